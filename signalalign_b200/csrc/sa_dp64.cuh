// FP64 cell arithmetic of the banded pair-HMM, shared by the plain one-read-per-launch kernel.
// Every formula keeps the reference's evaluation order (compile with -fmad=false) so results match
// signalAlign's CPU code to the last few ulps; only log()/exp() come from CUDA's math library.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sa {
namespace dp64 {

constexpr double kNegInf = -__builtin_huge_val();

struct Model64 {
    int32_t emission;            // sa_emission
    int32_t pad;
    double t[9];                 // transitions, StateMachine3 order
    const double *match, *gapy, *gapx;
    const double *klog;          // per k-mer: log sd and log lambda of the match and gap-Y rows
                                 // (the device's own log of the table values, computed once)
    double scale, shift, var;
    int64_t grid_length;
    const double *grid, *density, *slope;
    const int64_t *kmer_row;
};

// lookup + logAdd (pairwiseAligner.c:237-254): log(e^x + e^y) by a 4-piece cubic in the difference,
// exact max once the difference reaches 7.5; float literals evaluated in double as in the reference.
// The piece's coefficients are selected, not branched to, and the cubic is evaluated in the
// reference's order, so results are the reference's bit for bit.
__device__ __forceinline__ double lookup(double d) {
    const bool p0 = d <= 1.00f, p1 = d <= 2.50f, p2 = d <= 4.50f;
    const double a = p0 ? (double) -0.009350833524763f : p1 ? (double) -0.014532321752540f
                   : p2 ? (double) -0.004605031767994f : (double) -0.000458661602210f;
    const double b = p0 ? (double) 0.130659527668286f : p1 ? (double) 0.139942324101744f
                   : p2 ? (double) 0.063427417320019f : (double) 0.009695946122598f;
    const double c = p0 ? (double) 0.498799810682272f : p1 ? (double) 0.495635523139337f
                   : p2 ? (double) 0.695956496475118f : (double) 0.930734667215156f;
    const double e = p0 ? (double) 0.693203116424741f : p1 ? (double) 0.692140569840976f
                   : p2 ? (double) 0.514272634594009f : (double) 0.168037164329057f;
    return ((a * d + b) * d + c) * d + e;
}

__device__ __forceinline__ double log_add(double x, double y) {
    const bool lt = x < y;
    const double hi = lt ? y : x, lo = lt ? x : y;
    return (lo == kNegInf || hi - lo >= 7.5) ? hi : lookup(hi - lo) + lo;
}

// emissions_signal_descaleEventMean_JordanStyle (stateMachine.c:285-289)
__device__ __forceinline__ double descale(double e, double mu, double scale, double shift, double var) {
    return (e + var * mu - scale * mu - shift) / var;
}

// grid_spline_interp (hdp_math_utils.c:471-495) on the k-mer's density row
__device__ __forceinline__ double grid_spline(const Model64 &M, const double *y, const double *s, double q) {
    const double *x = M.grid;
    const int64_t len = M.grid_length;
    if (q <= x[0]) return y[0] - s[0] * (x[0] - q);
    if (q >= x[len - 1]) return y[len - 1] + s[len - 1] * (q - x[len - 1]);
    double dx = x[1] - x[0];
    int64_t il = (int64_t) ((q - x[0]) / dx);
    if (il > len - 2) il = len - 2;   // q just below the last knot can round onto it
    if (il < 0) il = 0;
    const int64_t ir = il + 1;
    double dy = y[ir] - y[il];
    double a = s[il] * dx - dy;
    double b = dy - s[ir] * dx;
    double tl = (q - x[il]) / dx;
    double tr = 1.0 - tl;
    return tr * y[il] + tl * y[ir] + tl * tr * (a * tr + b * tl);
}

// match (match=true) or extra-event emission of event (mean, noise) by k-mer kid:
// strawMan...WithDescaling / strawMan... (stateMachine.c:498-589) or getHdpKmerDensity (:468-495)
__device__ __forceinline__ double emit_event(const Model64 &M, int32_t kid, double mean, double noise, bool match) {
    if (kid < 0) return kNegInf;
    if (M.emission == 2) {
        double mu = M.match[(int64_t) kid * 5];
        double u = descale(mean, mu, M.scale, M.shift, M.var);
        int64_t row = M.kmer_row[kid];
        double d = row < 0 ? 0.0 : grid_spline(M, M.density + row * M.grid_length, M.slope + row * M.grid_length, u);
        if (!(d > 0.0)) d = 0.0;
        return log((1 / M.var) * d);
    }
    const double *tab = (match ? M.match : M.gapy) + (int64_t) kid * 5;
    const double *lg = M.klog + 4 * (int64_t) kid;
    double mu = tab[0], sd = tab[1];
    double m = M.emission == 1 ? descale(mean, mu, M.scale, M.shift, M.var) : mean;
    // emissions_signal_logGaussPdf and logInvGaussPdf (stateMachine.c:226-247), the logs of the
    // table's sd and lambda looked up
    double lm = kNegInf;
    if (sd != 0.0) {
        double a = (m - mu) / sd;
        lm = -0.91893853320467267 - lg[match ? 0 : 1] + (-0.5 * a * a);
    }
    const double nmu = tab[2], lambda = tab[4];
    double ln_n = log(noise);
    double b = (noise - nmu) / nmu;
    double ln = (lg[match ? 2 : 3] - 1.8378770664093453 - 3 * ln_n - lambda * b * b / noise) / 2;
    return lm + ln;
}

// emissions_kmer_getGapProb (stateMachine.c:155-172); the HDP machine uses log(0.1) (:1282)
__device__ __forceinline__ double emit_gapx(const Model64 &M, int32_t kid) {
    if (M.emission == 2) return -2.3025850929940455;
    if (kid < 0) return kNegInf;
    return M.gapx[kid];
}

}  // namespace dp64
}  // namespace sa
