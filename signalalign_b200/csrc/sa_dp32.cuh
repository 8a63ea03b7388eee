// FP32 cell arithmetic of the batched form.
//
// Values are log probabilities kept relative to a per-anti-diagonal base (an FP64 offset carried
// alongside), so the FP32 numbers stay within a few tens of zero and keep ~1e-6 absolute accuracy.
// logAdd is the reference's own 4-piece cubic (pairwiseAligner.c:237-254) evaluated in FP32: the
// reference's posteriors depend on that approximation at the 1e-3 level, so an exact log-sum-exp
// would not reproduce them.  The cubic is shift-invariant, so working relative to a base changes
// nothing but rounding.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sa_internal.h"

namespace sa {
namespace dp32 {

constexpr float kNegInf = -__builtin_huge_valf();

// the four cubic pieces of lookup() as float4 (a3, a2, a1, a0): p(d) = ((a3 d + a2) d + a1) d + a0
struct LogAddTable {
    float4 c[4];
};

__host__ __device__ constexpr LogAddTable log_add_table() {
    return LogAddTable{{
        {-0.009350833524763f, 0.130659527668286f, 0.498799810682272f, 0.693203116424741f},
        {-0.014532321752540f, 0.139942324101744f, 0.495635523139337f, 0.692140569840976f},
        {-0.004605031767994f, 0.063427417320019f, 0.695956496475118f, 0.514272634594009f},
        {-0.000458661602210f, 0.009695946122598f, 0.930734667215156f, 0.168037164329057f}}};
}

// logAdd with the cubic pieces read from shared memory (conflict-free: the four float4 occupy
// distinct banks).  Returns the larger argument when the difference reaches 7.5 or the smaller
// argument is -inf (both -inf gives NaN difference and also returns the max, -inf).
__device__ __forceinline__ float log_add(const float4 *tab, float x, float y) {
    const float mx = fmaxf(x, y), mn = fminf(x, y);
    const float d = mx - mn;
    const int seg = (d > 1.0f) + (d > 2.5f) + (d > 4.5f);
    const float4 c = tab[seg];
    const float p = fmaf(fmaf(fmaf(c.x, d, c.y), d, c.z), d, c.w);
    return d < 7.5f ? p + mn : mx;
}

// per-event FP32 record prepared on the device from the FP64 (mean, noise): mean, noise,
// -1.5*log(noise), 1/noise
struct __align__(16) Event32 {
    float mean, noise, c_noise, inv_noise;
};

// Gaussian level + inverse-Gaussian noise emissions of the match and extra-event states for one
// (k-mer, event):  log N(descaled mean; mu, sd) + log IG(noise; nu, lambda), with the extra-event
// state using sd x 1.75 (stateMachine.c:498-545, :226-247, :285-289).  The descaled residual is
// (mean - scale*mu - shift) / var.  kp: per-k-mer constants from the host.
struct ReadScale32 {
    float scale, shift, inv_var, log_inv_var;
};

__device__ __forceinline__ void emit_gauss(const KmerConst32 &k, const Event32 &ev, const ReadScale32 &rs,
                                           float &e_match, float &e_gapy) {
    const float r = (ev.mean - fmaf(rs.scale, k.mu, rs.shift)) * rs.inv_var;
    const float am = r * k.inv_sd_m, ay = r * k.inv_sd_y;
    const float b = fmaf(ev.noise, k.inv_nu, -1.0f);
    const float common = fmaf(-k.half_lambda, b * b * ev.inv_noise, ev.c_noise);
    e_match = fmaf(-0.5f * am, am, k.k_m + common);
    e_gapy = fmaf(-0.5f * ay, ay, k.k_y + common);
}

}  // namespace dp32
}  // namespace sa
