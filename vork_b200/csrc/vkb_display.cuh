// Display stage: linear Rec.709 RGBA (the resolved mean image) -> display code values,
// quantised like the resolve stage's unorm store.  The view is vork's std/standard
// (libraries/std/standard.slang:1-33): exposure, the sRGB transfer, a creative gamma on
// the code values, and for wider destinations the Display P3 or Rec.2020 primaries with
// the sRGB, ST 2084 or BT.2100 HLG encodings of libraries/std/view.slang:3-25.
#pragma once
#include <stdint.h>

namespace vkb {

struct DisplayParams {
    uint32_t display, bits, unassociate;
    float exposure_scale, inv_gamma, peak, white, hlg_gamma;
};

__device__ __forceinline__ float srgb_encode(float c) { return c > .0031308f ? 1.055f * powf(fmaxf(c, 0.f), 1.f / 2.4f) - .055f : 12.92f * c; }
__device__ __forceinline__ float srgb_decode(float c) { return c > .04045f ? powf(fmaxf((c + .055f) / 1.055f, 0.f), 2.4f) : c / 12.92f; }
__device__ __forceinline__ float pq_encode(float nits) {
    const float l = powf(fmaxf(nits, 0.f) / 10000.f, .1593017578125f);
    return powf((.8359375f + 18.8515625f * l) / (1.f + 18.6875f * l), 78.84375f);
}
__device__ __forceinline__ float hlg_oetf(float e) {
    return e <= 1.f / 12.f ? sqrtf(3.f * fmaxf(e, 0.f)) : .17883277f * logf(fmaxf(12.f * e - .28466892f, .000001f)) + .55991073f;
}

// std/standard for one pixel: linear Rec.709 -> code values of the destination.
__device__ __forceinline__ float3 standard_view(float3 c, const DisplayParams& d) {
    c = make_float3(c.x * d.exposure_scale, c.y * d.exposure_scale, c.z * d.exposure_scale);
    float3 m = make_float3(srgb_encode(c.x), srgb_encode(c.y), srgb_encode(c.z));
    if (d.display == 0u) {   // sRGB: the codes, with the creative gamma on them
        if (d.inv_gamma != 1.f) m = make_float3(powf(fmaxf(m.x, 0.f), d.inv_gamma), powf(fmaxf(m.y, 0.f), d.inv_gamma), powf(fmaxf(m.z, 0.f), d.inv_gamma));
        return m;
    }
    if (d.inv_gamma != 1.f)
        c = make_float3(srgb_decode(powf(fmaxf(m.x, 0.f), d.inv_gamma)), srgb_decode(powf(fmaxf(m.y, 0.f), d.inv_gamma)),
                        srgb_decode(powf(fmaxf(m.z, 0.f), d.inv_gamma)));
    if (d.display == 1u)     // Display P3 primaries, sRGB transfer
        return make_float3(srgb_encode(.82246197f * c.x + .17753803f * c.y),
                           srgb_encode(.03319420f * c.x + .96680580f * c.y),
                           srgb_encode(.01708263f * c.x + .07239744f * c.y + .91051993f * c.z));
    // Rec.2100: Rec.2020 primaries, unit white at the reference white, limited to the peak.
    float3 n = make_float3(.62740390f * c.x + .32928304f * c.y + .04331307f * c.z, .06909729f * c.x + .91954040f * c.y + .01136232f * c.z,
                           .01639144f * c.x + .08801331f * c.y + .89559525f * c.z);
    n = make_float3(fminf(fmaxf(n.x * d.white, 0.f), d.peak), fminf(fmaxf(n.y * d.white, 0.f), d.peak), fminf(fmaxf(n.z * d.white, 0.f), d.peak));
    if (d.display == 2u) return make_float3(pq_encode(n.x), pq_encode(n.y), pq_encode(n.z));
    // HLG: inverse OOTF with the system gamma for the peak, then the OETF.
    const float3 l = make_float3(n.x / d.peak, n.y / d.peak, n.z / d.peak);
    const float y = fmaxf(.2627f * l.x + .6780f * l.y + .0593f * l.z, 1e-4f / powf(3.f, d.hlg_gamma));
    const float s = powf(y, (1.f - d.hlg_gamma) / d.hlg_gamma);
    return make_float3(hlg_oetf(l.x * s), hlg_oetf(l.y * s), hlg_oetf(l.z * s));
}

// One pixel per thread: view, then unorm quantisation round(saturate(v) * (2^bits - 1))
// (resolve.slang:13) or float codes (bits 32).  Non-finite input sets *nonfinite.
__global__ void k_display(uint32_t n, const float4* __restrict__ rgba, DisplayParams d, void* __restrict__ out, uint32_t* nonfinite) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p = rgba[i];
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(p.w))) {
            atomicOr(nonfinite, 1u);
            p = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float3 c = make_float3(p.x, p.y, p.z);
        if (d.unassociate && p.w > 0.f) c = make_float3(c.x / p.w, c.y / p.w, c.z / p.w);   // resolve.slang:140-145
        const float3 v = standard_view(c, d);
        const float q[4] = {v.x, v.y, v.z, p.w};
        if (d.bits == 8u) {
            uchar4 o;
            unsigned char* b = &o.x;
            for (int k = 0; k < 4; ++k) b[k] = (unsigned char)rintf(fminf(fmaxf(q[k], 0.f), 1.f) * 255.f);
            static_cast<uchar4*>(out)[i] = o;
        } else if (d.bits == 16u) {
            ushort4 o;
            unsigned short* b = &o.x;
            for (int k = 0; k < 4; ++k) b[k] = (unsigned short)rintf(fminf(fmaxf(q[k], 0.f), 1.f) * 65535.f);
            static_cast<ushort4*>(out)[i] = o;
        } else {
            static_cast<float4*>(out)[i] = make_float4(q[0], q[1], q[2], q[3]);
        }
    }
}

}  // namespace vkb
