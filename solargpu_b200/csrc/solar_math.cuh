// Device helpers shared by the solar and reflection kernels.
#pragma once

#include "sgb_internal.cuh"

namespace sgb {

// Direct + Perez diffuse of one voxel for one daylight hour
// (src/cuda/kernels/solar_kernel.cu:54-77 with the per-hour terms hoisted):
//   cos_aoi = cos z cos s + sin z sin s cos(az - aspect) = dot(n, s_h)
//   direct  = max(0, max(DNI, 1e-3) * cos_aoi) when cos_aoi > 0, the hour has
//             a sun bin and the voxel's shadow bit for it is clear
//   diffuse = DHI ((1 - F1)(1 + cos s)/2 + F1 max(0, cos_aoi)/b + F2 sin s)
// n = (sin s sin a, -sin s cos a, cos s), n4.w = sin s.
__device__ __forceinline__ float solar_I(const float4 n4, const HourEntry& e, uint32_t shadow_bit)
{
    const float caoi = fmaf(n4.x, e.sx, fmaf(n4.y, e.sy, n4.z * e.sz));
    float I = 0.0f;
    if (caoi > 0.0f && e.dense >= 0 && !shadow_bit) I = fmaxf(0.0f, e.dni_eff * caoi);
    const float dif = fmaf(e.c0, 1.0f + n4.z, fmaf(e.c1, fmaxf(0.0f, caoi), e.c2 * n4.w));
    return I + fmaxf(0.0f, dif);
}

__device__ __forceinline__ uint32_t shadow_bit(const uint32_t* __restrict__ shadow, int words32,
                                               long long v, int dense)
{
    if (dense < 0) return 0u;
    return (__ldg(shadow + v * words32 + (dense >> 5)) >> (dense & 31)) & 1u;
}

// Inter-reflection weight of top cell `nb` toward receiver `me`
// (src/cuda/kernels/reflection_kernels.cu:18-38, hour-independent part):
//   w = albedo * cos_recv * cos_send / (pi d^2), 0 if d^2 < 1e-4 or cos_recv <= 0,
//   cos_send = max(|dz| / d, 0.1).
__device__ __forceinline__ float refl_weight(const float4 me_p, const float4 me_n, const float4 nb_p)
{
    const float dx = nb_p.x - me_p.x;
    const float dy = nb_p.y - me_p.y;
    const float dz = nb_p.z - me_p.z;
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (d2 < 1e-4f) return 0.0f;
    const float dot = fmaf(me_n.x, dx, fmaf(me_n.y, dy, me_n.z * dz));
    if (dot <= 0.0f) return 0.0f;
    const float inv = rsqrtf(d2);
    const float crecv = dot * inv;
    const float csend = fmaxf(fabsf(dz) * inv, 0.1f);
    // kAlbedo / pi with the reference's constants (0.2f, 3.14159265f)
    return (0.2f / 3.14159265f) * crecv * csend * (inv * inv);
}

}  // namespace sgb
