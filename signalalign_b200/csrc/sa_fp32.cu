// Batched FP32 form: all regions of all reads in one persistent launch.
//
// Work distribution: regions are sorted by band area (largest first) on the host; persistent CTAs
// of 128 threads pull the next region from a device counter.  A CTA sweeps its region's band one
// anti-diagonal at a time (cells of an anti-diagonal spread over the threads, neighbours exchanged
// through a 3-slot shared-memory ring, one barrier per anti-diagonal).  Forward values go to HBM
// (3 floats per cell, SoA per anti-diagonal) together with each anti-diagonal's FP64 base.  At each
// traceback point of getPosteriorProbsWithBanding (pairwiseAligner.c:1319-1333) the CTA runs the
// window's backward sweep in shared memory with the posterior test fused into it, so backward
// values never leave the SM.  Total probabilities are refreshed on the reference's schedule
// (every 10th posterior anti-diagonal, :1370-1380) and accumulated in the reference's sequential
// cell order, which the 7.5 cut-off of logAdd makes order dependent.
//
// Values are log probabilities relative to a per-anti-diagonal base: the base of anti-diagonal d is
// the base of d-1 plus the largest value stored on d-1 (FP64, carried by every thread), so stored
// FP32 values stay near zero.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "sa_dp32.cuh"
#include "sa_internal.h"

namespace sa {
namespace fp32 {

using namespace dp32;

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;

enum { T_MC = 0, T_MFGX, T_MFGY, T_OX, T_OY, T_EX, T_EY, T_SX, T_SY };

struct ModelDesc {
    const KmerConst32 *kc;
    const float *gapx;
    Hdp32 hdp;
    int32_t emission;
    int32_t pad;
    float t[9];
    float pad2;
};

struct RegionDesc {
    int32_t n, lX, lY, read;
    int32_t n_windows, model;
    int32_t ragged_left, ragged_right;
    int64_t diag_base;    // first anti-diagonal of this region in the per-anti-diagonal arrays
    int64_t cell_base;    // first cell of this region in the forward store
    int64_t win_base;
    int64_t kmer_base;    // k-mer id of column x >= 1 is kmer[kmer_base + x - 1]
    int64_t event_base;   // event of row y >= 1 is events[event_base + y - 1]
    int64_t out_base, out_cap;
    int64_t x1, y1;
};

struct Args {
    const RegionDesc *regions;
    const int32_t *order;
    int64_t n_regions;
    const ModelDesc *models;
    const ReadScale32 *read_scale;
    const int32_t *xl, *xr;        // per anti-diagonal band
    const int64_t *coff;           // per anti-diagonal first cell (region-relative)
    const Window *windows;
    const int32_t *kmer;
    const Event32 *events;
    float *F;                      // forward store
    double *base;                  // per anti-diagonal FP64 base of the forward store
    float *fmax;                   // per anti-diagonal largest stored forward value
    sa_aligned_pair *out;
    int64_t *out_count;            // per region
    double *loglik;                // per region: total probability at its last anti-diagonal
    int32_t *status;               // per read
    unsigned int *queue;
    float threshold;
    int32_t cpt;                   // cells per thread
};

struct Shared {
    float4 la[4];
    float wmax[2][kWarps];
    int32_t wcnt[8][kWarps];
    float pval;
};

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sequential logAdd over vals[0..n) in index order, exactly as a one-thread loop would fold it
// (dpDiagonal_dotProduct, pairwiseAligner.c:1014-1027), run by one warp: a value can only change the
// running result if it exceeds the running maximum minus 7.5 (the running result never falls below
// the running maximum), so only those values are folded, in order.
__device__ float ordered_fold(const float4 *tab, const float *vals, int n) {
    const int lane = threadIdx.x & 31;
    float r = kNegInf, carry = kNegInf;
    for (int b = 0; b < n; b += 32) {
        const float v = b + lane < n ? vals[b + lane] : kNegInf;
        float incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl = fmaxf(incl, t);
        }
        incl = fmaxf(incl, carry);
        float excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) excl = carry;
        unsigned mask = __ballot_sync(0xffffffffu, v > excl - 7.6f);
        while (mask) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1;
            r = log_add(tab, r, __shfl_sync(0xffffffffu, v, bit));
        }
        carry = __shfl_sync(0xffffffffu, incl, 31);
    }
    return r;
}

__global__ void prep_events(const double2 *raw, Event32 *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const double2 e = raw[i];
        Event32 v;
        v.mean = (float) e.x;
        v.noise = (float) e.y;
        v.c_noise = (float) (-1.5 * log(e.y));
        v.inv_noise = (float) (1.0 / e.y);
        out[i] = v;
    }
}

struct Ctx {
    const Args *A;
    RegionDesc Rv;
    const RegionDesc *R;   // points at Rv
    int32_t region_index;
    const ModelDesc *M;
    ReadScale32 rs;
    Shared *sh;
    float *fring;     // [3 slots][3 states][wmax]
    float *bring;     // [3 slots][3 states][wmax]
    float *chain;     // [2][wmax]
    int wmax;
};

__device__ __forceinline__ int32_t kmer_of(const Ctx &c, int32_t x) {
    return x > 0 ? __ldg(c.A->kmer + c.R->kmer_base + x - 1) : -1;
}

__device__ __forceinline__ void emissions(const Ctx &c, int32_t kid, int32_t y_event, float &em, float &ey) {
    const Event32 ev = c.A->events[c.R->event_base + y_event];
    if (kid < 0) { em = ey = kNegInf; return; }
    const KmerConst32 k = c.M->kc[kid];
    if (c.M->emission == SA_EMIT_HDP) {
        em = ey = emit_hdp(c.M->hdp, k, kid, ev, c.rs);
    } else {
        emit_gauss(k, ev, c.rs, em, ey);
    }
}

__device__ __forceinline__ float emission_gapx(const Ctx &c, int32_t kid) {
    if (c.M->emission == SA_EMIT_HDP) return (float) kLogPointOne;
    return kid < 0 ? kNegInf : __ldg(c.M->gapx + kid);
}

__device__ __forceinline__ float *ring(float *r, int wmax, int slot, int state) { return r + (slot * 3 + state) * wmax; }

// total probability of anti-diagonal d (diagonalCalculationTotalProbability, pairwiseAligner.c:
// 1182-1200) relative to base(F_d) + base(B_d).  fs/bs: slots of F_d (global) and B_d, B_{d+1} (ring).
__device__ float total_probability(Ctx &c, int32_t d, bool have_next, int slot_d, int slot_n, float fmax_prev,
                                   float bmax_next) {
    const Args &A = *c.A;
    const RegionDesc &R = *c.R;
    const float4 *tab = c.sh->la;
    const float *t = c.M->t;
    const int tid = threadIdx.x;
    const int32_t L = A.xl[R.diag_base + d], W = (A.xr[R.diag_base + d] - L) / 2 + 1;
    const float *Fd = A.F + 3 * (R.cell_base + A.coff[R.diag_base + d]);
    const float *bM = ring(c.bring, c.wmax, slot_d, 0), *bX = ring(c.bring, c.wmax, slot_d, 1),
                *bY = ring(c.bring, c.wmax, slot_d, 2);
    for (int i = tid; i < W; i += kThreads) {
        float s = Fd[i] + bM[i];
        s = log_add(tab, s, Fd[W + i] + bX[i]);
        s = log_add(tab, s, Fd[2 * W + i] + bY[i]);
        c.chain[i] = s;
    }
    int32_t Wn = 0;
    if (have_next && d >= 1) {
        const int32_t dn = d + 1;
        const int32_t Ln = A.xl[R.diag_base + dn];
        Wn = (A.xr[R.diag_base + dn] - Ln) / 2 + 1;
        const int32_t Lp = A.xl[R.diag_base + d - 1], Rp = A.xr[R.diag_base + d - 1];
        const int32_t Wp = (Rp - Lp) / 2 + 1;
        const float *Fp = A.F + 3 * (R.cell_base + A.coff[R.diag_base + d - 1]);
        const float *nM = ring(c.bring, c.wmax, slot_n, 0);
        const float shift = -fmax_prev - bmax_next;
        for (int i = tid; i < Wn; i += kThreads) {
            const int32_t xmy = Ln + 2 * i;
            float m = kNegInf;
            if (xmy >= Lp && xmy <= Rp) {
                const int32_t x = (dn + xmy) >> 1, y = (dn - xmy) >> 1;
                const int32_t im = (xmy - Lp) >> 1;
                float em, ey;
                emissions(c, kmer_of(c, x), y - 1, em, ey);
                m = Fp[im] + (em + t[T_MC]);
                m = log_add(tab, m, Fp[Wp + im] + (em + t[T_MFGX]));
                m = log_add(tab, m, Fp[2 * Wp + im] + (em + t[T_MFGY]));
            }
            c.chain[c.wmax + i] = m + nM[i] + shift;
        }
    }
    __syncthreads();
    if (tid < 32) {
        float p = ordered_fold(tab, c.chain, W);
        if (Wn > 0) p = log_add(tab, p, ordered_fold(tab, c.chain + c.wmax, Wn));
        if (tid == 0) c.sh->pval = p;
    }
    __syncthreads();
    return c.sh->pval;
}

__device__ void run_region(Ctx &c) {
    const Args &A = *c.A;
    const RegionDesc &R = *c.R;
    const ModelDesc &M = *c.M;
    const float *t = M.t;
    const float4 *tab = c.sh->la;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t db = R.diag_base;
    const int cpt = A.cpt;

    // anti-diagonal 0: startStateProb / raggedStartStateProb (stateMachine.c:1022-1032)
    if (tid == 0) {
        const float s0 = R.ragged_left ? kNegInf : 0.0f, s1 = R.ragged_left ? 0.0f : kNegInf;
        float *F0 = A.F + 3 * (R.cell_base + A.coff[db]);
        F0[0] = s0; F0[1] = s1; F0[2] = s1;
        ring(c.fring, c.wmax, 0, 0)[0] = s0;
        ring(c.fring, c.wmax, 0, 1)[0] = s1;
        ring(c.fring, c.wmax, 0, 2)[0] = s1;
        A.base[db] = 0.0;
        A.fmax[db] = 0.0f;
    }
    __syncthreads();
    double fbase = 0.0;        // base of the anti-diagonal being computed
    float m1 = 0.0f, m2 = 0.0f;  // largest stored value of anti-diagonals d-1, d-2
    int32_t Lp = A.xl[db], Rp = A.xr[db], Lpp = 0, Rpp = -1;
    int32_t wi = 0;
    Window W = A.windows[R.win_base];
    int64_t n_out = 0;
    double ll = 0.0;
    for (int32_t d = 1; d <= R.n; ++d) {
        fbase += (double) m1;
        const int32_t L = A.xl[db + d], Rr = A.xr[db + d], Wd = (Rr - L) / 2 + 1;
        const int slot = d % 3, s1 = (d + 2) % 3, s2 = (d + 1) % 3;
        float *Fd = A.F + 3 * (R.cell_base + A.coff[db + d]);
        float lmax = kNegInf;
        for (int j = 0; j < cpt; ++j) {
            const int i = tid + j * kThreads;
            if (i >= Wd) break;
            const int32_t xmy = L + 2 * i, x = (d + xmy) >> 1, y = (d - xmy) >> 1;
            const int32_t kid = kmer_of(c, x);
            float vM = kNegInf, vX = kNegInf, vY = kNegInf;
            const bool lower = xmy - 1 >= Lp && xmy - 1 <= Rp;
            const bool upper = xmy + 1 >= Lp && xmy + 1 <= Rp;
            const bool middle = d >= 2 && xmy >= Lpp && xmy <= Rpp;
            if (lower) {
                const int il = (xmy - 1 - Lp) >> 1;
                const float e = emission_gapx(c, kid) - m1;
                vX = ring(c.fring, c.wmax, s1, 0)[il] + (e + t[T_OX]);
                vX = log_add(tab, vX, ring(c.fring, c.wmax, s1, 1)[il] + (e + t[T_EX]));
                vX = log_add(tab, vX, ring(c.fring, c.wmax, s1, 2)[il] + (e + t[T_SX]));
            }
            if (middle || upper) {
                float em, ey;
                emissions(c, kid, y - 1, em, ey);
                if (middle) {
                    const int im = (xmy - Lpp) >> 1;
                    const float e = em - m2 - m1;
                    vM = ring(c.fring, c.wmax, s2, 0)[im] + (e + t[T_MC]);
                    vM = log_add(tab, vM, ring(c.fring, c.wmax, s2, 1)[im] + (e + t[T_MFGX]));
                    vM = log_add(tab, vM, ring(c.fring, c.wmax, s2, 2)[im] + (e + t[T_MFGY]));
                }
                if (upper) {
                    const int iu = (xmy + 1 - Lp) >> 1;
                    const float e = ey - m1;
                    vY = ring(c.fring, c.wmax, s1, 0)[iu] + (e + t[T_OY]);
                    vY = log_add(tab, vY, ring(c.fring, c.wmax, s1, 2)[iu] + (e + t[T_EY]));
                }
            }
            ring(c.fring, c.wmax, slot, 0)[i] = vM;
            ring(c.fring, c.wmax, slot, 1)[i] = vX;
            ring(c.fring, c.wmax, slot, 2)[i] = vY;
            Fd[i] = vM;
            Fd[Wd + i] = vX;
            Fd[2 * Wd + i] = vY;
            lmax = fmaxf(lmax, fmaxf(vM, fmaxf(vX, vY)));
        }
        lmax = warp_max(lmax);
        if (lane == 0) c.sh->wmax[d & 1][warp] = lmax;
        __syncthreads();
        float md = c.sh->wmax[d & 1][0];
#pragma unroll
        for (int w = 1; w < kWarps; ++w) md = fmaxf(md, c.sh->wmax[d & 1][w]);
        if (!(md > kNegInf)) md = 0.0f;
        if (tid == 0) {
            A.base[db + d] = fbase;
            A.fmax[db + d] = md;
        }
        m2 = m1; m1 = md;
        Lpp = Lp; Rpp = Rp; Lp = L; Rp = Rr;
        if (d != W.D) continue;

        // ---------------- backward sweep of the window (T, D] with fused posteriors -------------
        __threadfence_block();
        const bool ragged_end = W.at_end && R.ragged_right;
        const float e0 = ragged_end ? (t[T_OX] + t[T_OY]) / 2.0f : t[T_MC];
        const float e1 = ragged_end ? t[T_EX] : t[T_MFGX];
        const float e2 = ragged_end ? t[T_EY] : t[T_MFGY];
        {
            const int sl = d % 3;
            for (int i = tid; i < Wd; i += kThreads) {
                ring(c.bring, c.wmax, sl, 0)[i] = e0;
                ring(c.bring, c.wmax, sl, 1)[i] = e1;
                ring(c.bring, c.wmax, sl, 2)[i] = e2;
            }
        }
        float bm_end = fmaxf(e0, fmaxf(e1, e2));
        if (!(bm_end > kNegInf)) bm_end = 0.0f;
        double bbase = 0.0;            // base of B on the anti-diagonal being processed
        float b1 = bm_end, b2 = 0.0f;  // largest stored B value on d2+1, d2+2
        int32_t BLn = L, BRn = Rr, BLnn = 0, BRnn = -1;   // band of d2+1, d2+2
        double pref = 0.0;             // latest refresh total probability (absolute)
        int32_t k = 0;
        __syncthreads();
        for (int32_t d2 = W.D; d2 > W.T; --d2) {
            const int sl = d2 % 3, sn = (d2 + 1) % 3, snn = (d2 + 2) % 3;
            const int32_t BL = A.xl[db + d2], BR = A.xr[db + d2], BW = (BR - BL) / 2 + 1;
            float bmd = bm_end;
            if (d2 < W.D) {
                bbase += (double) b1;
                float lm = kNegInf;
                for (int j = 0; j < cpt; ++j) {
                    const int i = tid + j * kThreads;
                    if (i >= BW) break;
                    const int32_t xmy = BL + 2 * i, x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
                    float vM = kNegInf, vX = kNegInf, vY = kNegInf;
                    const bool mid = d2 + 2 <= W.D && xmy >= BLnn && xmy <= BRnn;
                    const bool up = xmy - 1 >= BLn && xmy - 1 <= BRn;
                    const bool lo = xmy + 1 >= BLn && xmy + 1 <= BRn;
                    if (mid) {
                        float em, ey;
                        emissions(c, kmer_of(c, x + 1), y, em, ey);
                        const float bmv = ring(c.bring, c.wmax, snn, 0)[(xmy - BLnn) >> 1];
                        const float e = em - b2 - b1;
                        vM = bmv + (e + t[T_MC]);
                        vX = bmv + (e + t[T_MFGX]);
                        vY = bmv + (e + t[T_MFGY]);
                    }
                    if (up) {
                        float em, ey;
                        emissions(c, kmer_of(c, x), y, em, ey);
                        const float buv = ring(c.bring, c.wmax, sn, 2)[(xmy - 1 - BLn) >> 1];
                        const float e = ey - b1;
                        vM = log_add(tab, vM, buv + (e + t[T_OY]));
                        vY = log_add(tab, vY, buv + (e + t[T_EY]));
                    }
                    if (lo) {
                        const float blv = ring(c.bring, c.wmax, sn, 1)[(xmy + 1 - BLn) >> 1];
                        const float e = emission_gapx(c, kmer_of(c, x + 1)) - b1;
                        vM = log_add(tab, vM, blv + (e + t[T_OX]));
                        vX = log_add(tab, vX, blv + (e + t[T_EX]));
                        vY = log_add(tab, vY, blv + (e + t[T_SX]));
                    }
                    ring(c.bring, c.wmax, sl, 0)[i] = vM;
                    ring(c.bring, c.wmax, sl, 1)[i] = vX;
                    ring(c.bring, c.wmax, sl, 2)[i] = vY;
                    lm = fmaxf(lm, fmaxf(vM, fmaxf(vX, vY)));
                }
                lm = warp_max(lm);
                if (lane == 0) c.sh->wmax[d2 & 1][warp] = lm;
                __syncthreads();
                bmd = c.sh->wmax[d2 & 1][0];
#pragma unroll
                for (int w = 1; w < kWarps; ++w) bmd = fmaxf(bmd, c.sh->wmax[d2 & 1][w]);
                if (!(bmd > kNegInf)) bmd = 0.0f;
            }
            if (d2 <= W.from) {
                const double fb = A.base[db + d2];
                if (k++ % 10 == 0) {
                    const bool have_next = d2 < W.D;
                    const float fmp = d2 >= 1 ? A.fmax[db + d2 - 1] : 0.0f;
                    const float pt = total_probability(c, d2, have_next, sl, sn, fmp, b1);
                    pref = (double) pt + fb + bbase;
                    if (d2 == R.n) ll = pref;
                }
                const float kd = (float) (fb + bbase - pref);
                const float *Fm = A.F + 3 * (R.cell_base + A.coff[db + d2]);
                const float *bM = ring(c.bring, c.wmax, sl, 0);
                unsigned flags = 0;
                float pv[8];
                for (int j = 0; j < cpt && j < 8; ++j) {
                    const int i = tid + j * kThreads;
                    pv[j] = 0.0f;
                    if (i < BW) {
                        const int32_t xmy = BL + 2 * i, x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
                        if (x > 0 && y > 0) {
                            const float p = __expf(Fm[i] + bM[i] + kd);
                            if (p >= A.threshold) { flags |= 1u << j; pv[j] = p; }
                        }
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, (flags >> j) & 1u);
                    if (lane == 0) c.sh->wcnt[j][warp] = __popc(bal);
                }
                __syncthreads();
                int64_t before = 0;
                for (int j = 0; j < cpt && j < 8; ++j) {
                    int32_t tot = 0, pre = 0;
#pragma unroll
                    for (int w = 0; w < kWarps; ++w) {
                        const int32_t cw = c.sh->wcnt[j][w];
                        if (w < warp) pre += cw;
                        tot += cw;
                    }
                    const unsigned mine = __ballot_sync(0xffffffffu, (flags >> j) & 1u);
                    if ((flags >> j) & 1u) {
                        const int rank = __popc(mine & ((1u << lane) - 1u));
                        const int64_t slot64 = n_out + before + pre + rank;
                        const int i = tid + j * kThreads;
                        const int32_t xmy = BL + 2 * i, x = (d2 + xmy) >> 1, y = (d2 - xmy) >> 1;
                        if (slot64 < R.out_cap) {
                            sa_aligned_pair o;
                            const float p = fminf(pv[j], 1.0f);
                            o.score = (int64_t) floor((double) p * 10000000.0);
                            o.x = R.x1 + x - 1;
                            o.y = R.y1 + y - 1;
                            o.kmer = kmer_of(c, x);
                            A.out[R.out_base + slot64] = o;
                        } else {
                            atomicMax(A.status + R.read, (int32_t) SA_E_OUTPUT);
                        }
                    }
                    before += tot;
                }
                n_out += before;
            }
            b2 = b1; b1 = bmd;
            BLnn = BLn; BRnn = BRn; BLn = BL; BRn = BR;
        }
        __syncthreads();
        if (W.at_end) break;
        W = A.windows[R.win_base + (++wi)];
    }
    if (tid == 0) {
        A.out_count[c.region_index] = n_out;
        A.loglik[c.region_index] = ll;
    }
}

__global__ void __launch_bounds__(kThreads) batch_kernel(const __grid_constant__ Args A, int wmax) {
    extern __shared__ float4 smem_raw[];
    Shared *sh = reinterpret_cast<Shared *>(smem_raw);
    float *fring = reinterpret_cast<float *>(sh + 1);
    float *bring = fring + 9 * wmax;
    float *chain = bring + 9 * wmax;
    if (threadIdx.x < 4) {
        const LogAddTable lt = log_add_table();
        sh->la[threadIdx.x] = lt.c[threadIdx.x];
    }
    __shared__ int32_t next;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) next = (int32_t) atomicAdd(A.queue, 1u);
        __syncthreads();
        const int32_t qi = next;
        if (qi >= A.n_regions) break;
        Ctx c;
        c.A = &A;
        c.region_index = A.order[qi];
        c.Rv = A.regions[c.region_index];
        c.R = &c.Rv;
        c.M = A.models + c.Rv.model;
        c.rs = A.read_scale[c.R->read];
        c.sh = sh;
        c.fring = fring;
        c.bring = bring;
        c.chain = chain;
        c.wmax = wmax;
        run_region(c);
    }
}

// FP32 issue-rate probe for the roofline denominator: 8 independent FMA chains per thread.
__global__ void __launch_bounds__(256) fma_probe(float *sink, int iters, float seed) {
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = seed + threadIdx.x * 1e-7f + i;
    const float m = 0.999999f, c = 1e-7f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], m, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 12345.678f) sink[0] = s;
}

}  // namespace fp32
}  // namespace sa

// ------------------------------------------------------------------------------------------------
// host side of the batch
// ------------------------------------------------------------------------------------------------
using namespace sa;
using namespace sa::fp32;

struct sa_batch {
    int device = 0;
    int64_t n_reads = 0;
    std::vector<sa_state_machine *> models;
    std::vector<RegionDesc> regions;
    std::vector<int32_t> order;
    std::vector<int32_t> read_status;       // host planning status per read
    std::vector<int64_t> read_first_region, read_n_regions;
    std::vector<ReadScale32> read_scale;
    std::vector<int32_t> xl, xr;
    std::vector<int64_t> coff;
    std::vector<Window> windows;
    std::vector<int32_t> kmer;
    std::vector<double2> events;
    int64_t cells = 0, out_total = 0;
    int32_t max_width = 0;
    float threshold = 0.01f;
    // device
    RegionDesc *d_regions = nullptr;
    int32_t *d_order = nullptr;
    ModelDesc *d_models = nullptr;
    ReadScale32 *d_read_scale = nullptr;
    int32_t *d_xl = nullptr, *d_xr = nullptr, *d_kmer = nullptr, *d_status = nullptr;
    int64_t *d_coff = nullptr, *d_out_count = nullptr;
    Window *d_windows = nullptr;
    double2 *d_events_raw = nullptr;
    Event32 *d_events = nullptr;
    float *d_F = nullptr, *d_fmax = nullptr;
    double *d_base = nullptr, *d_loglik = nullptr;
    sa_aligned_pair *d_out = nullptr;
    unsigned int *d_queue = nullptr;
    // results
    std::vector<int64_t> out_count;
    std::vector<double> loglik;
    std::vector<int32_t> dev_status;
    std::vector<sa_aligned_pair> out;
    std::vector<std::vector<sa_aligned_pair>> read_pairs;
    std::vector<double> read_ll;
    bool downloaded = false;
};

namespace {

template <typename T>
sa_status dalloc(T **p, size_t n) {
    if (n == 0) n = 1;
    return cudaMalloc((void **) p, n * sizeof(T)) == cudaSuccess ? SA_OK : SA_E_NOMEM;
}

template <typename T>
sa_status h2d(T *dst, const std::vector<T> &src, cudaStream_t s) {
    if (src.empty()) return SA_OK;
    return cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess
               ? SA_OK : SA_E_CUDA;
}

void free_batch_device(sa_batch *b) {
    cudaFree(b->d_regions); cudaFree(b->d_order); cudaFree(b->d_models); cudaFree(b->d_read_scale);
    cudaFree(b->d_xl); cudaFree(b->d_xr); cudaFree(b->d_kmer); cudaFree(b->d_status); cudaFree(b->d_coff);
    cudaFree(b->d_out_count); cudaFree(b->d_windows); cudaFree(b->d_events_raw); cudaFree(b->d_events);
    cudaFree(b->d_F); cudaFree(b->d_fmax); cudaFree(b->d_base); cudaFree(b->d_loglik); cudaFree(b->d_out);
    cudaFree(b->d_queue);
}

}  // namespace

extern "C" {

sa_status sa_batch_create(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch **out) {
    if (!reads || n_reads < 0 || !p || !out) return SA_E_ARG;
    *out = nullptr;
    sa_status st = check_params(*p);
    if (st) return st;
    auto *b = new (std::nothrow) sa_batch();
    if (!b) return SA_E_NOMEM;
    b->n_reads = n_reads;
    b->threshold = (float) p->threshold;
    b->read_status.assign(n_reads, SA_OK);
    b->read_first_region.assign(n_reads, 0);
    b->read_n_regions.assign(n_reads, 0);
    b->read_scale.resize(n_reads);
    std::vector<Region> regs;
    PathTable pt;
    int device = -1;
    for (int64_t r = 0; r < n_reads; ++r) {
        const sa_read &rd = reads[r];
        auto *sm = const_cast<sa_state_machine *>(rd.sm);
        b->read_first_region[r] = (int64_t) b->regions.size();
        if (!sm || rd.reference_length < 0 || rd.n_events < 0 || rd.n_anchors < 0 ||
            (rd.reference_length > 0 && !rd.reference) || (rd.n_events > 0 && !rd.events) ||
            (rd.n_anchors > 0 && !rd.anchors) || !(rd.var != 0.0)) {
            b->read_status[r] = SA_E_ARG;
            continue;
        }
        if (device < 0) device = sm->dev.device;
        if (sm->dev.device != device) { b->read_status[r] = SA_E_ARG; continue; }
        if (sm->emission == SA_EMIT_HDP && !sm->hdp.present) { b->read_status[r] = SA_E_UNSUPPORTED; continue; }
        const int k = sm->kmer_length;
        const int64_t lX = rd.reference_length == 0 ? 0 : rd.reference_length - (k - 1);
        if (lX < 0) { b->read_status[r] = SA_E_ARG; continue; }
        st = build_paths(sm, rd.reference, lX, rd.degenerate, pt);
        if (st) { b->read_status[r] = st; continue; }
        if (pt.multi) { b->read_status[r] = SA_E_UNSUPPORTED; continue; }
        st = plan_regions(rd.anchors, rd.n_anchors, lX, rd.n_events, *p, rd.ragged_left != 0, rd.ragged_right != 0,
                          regs);
        if (st) { b->read_status[r] = st; continue; }
        int32_t model = -1;
        for (size_t i = 0; i < b->models.size(); ++i)
            if (b->models[i] == sm) model = (int32_t) i;
        if (model < 0) { model = (int32_t) b->models.size(); b->models.push_back(sm); }
        const double var = sm->emission == SA_EMIT_PLAIN ? 1.0 : rd.var;
        ReadScale32 &rs = b->read_scale[r];
        rs.scale = sm->emission == SA_EMIT_PLAIN ? 1.0f : (float) rd.scale;
        rs.shift = sm->emission == SA_EMIT_PLAIN ? 0.0f : (float) rd.shift;
        rs.inv_var = (float) (1.0 / var);
        rs.log_inv_var = (float) std::log(1.0 / var);
        const int64_t kmer_base = (int64_t) b->kmer.size();
        for (int64_t x = 1; x <= lX; ++x) b->kmer.push_back(pt.ids[pt.first[x]]);
        const int64_t event_base = (int64_t) b->events.size();
        for (int64_t y = 0; y < rd.n_events; ++y)
            b->events.push_back(make_double2(rd.events[y * kEventParams], rd.events[y * kEventParams + 1]));
        for (const Region &rg : regs) {
            RegionDesc d;
            std::memset(&d, 0, sizeof(d));
            d.n = (int32_t) (rg.lX + rg.lY);
            d.lX = (int32_t) rg.lX;
            d.lY = (int32_t) rg.lY;
            d.read = (int32_t) r;
            d.n_windows = (int32_t) rg.windows.size();
            d.model = model;
            d.ragged_left = rg.ragged_left;
            d.ragged_right = rg.ragged_right;
            d.diag_base = (int64_t) b->xl.size();
            d.cell_base = b->cells;
            d.win_base = (int64_t) b->windows.size();
            d.kmer_base = kmer_base + rg.x1;
            d.event_base = event_base + rg.y1;
            d.x1 = rg.x1;
            d.y1 = rg.y1;
            d.out_cap = 4 * (int64_t) d.n + 256;
            d.out_base = b->out_total;
            b->out_total += d.out_cap;
            int64_t acc = 0;
            for (int32_t dd = 0; dd <= d.n; ++dd) {
                b->xl.push_back(rg.xmy_l[dd]);
                b->xr.push_back(rg.xmy_r[dd]);
                b->coff.push_back(acc);
                acc += (rg.xmy_r[dd] - rg.xmy_l[dd]) / 2 + 1;
            }
            b->cells += acc;
            b->max_width = std::max(b->max_width, rg.max_width);
            b->windows.insert(b->windows.end(), rg.windows.begin(), rg.windows.end());
            b->regions.push_back(d);
        }
        b->read_n_regions[r] = (int64_t) b->regions.size() - b->read_first_region[r];
    }
    if (b->max_width > 8 * kThreads) {
        delete b;
        return SA_E_CAPACITY;
    }
    b->device = device < 0 ? 0 : device;
    // largest band area first (LPT order for the persistent CTAs)
    b->order.resize(b->regions.size());
    std::iota(b->order.begin(), b->order.end(), 0);
    std::vector<int64_t> area(b->regions.size());
    for (size_t i = 0; i < b->regions.size(); ++i) {
        const RegionDesc &d = b->regions[i];
        area[i] = (i + 1 < b->regions.size() ? b->regions[i + 1].cell_base : b->cells) - d.cell_base;
    }
    std::stable_sort(b->order.begin(), b->order.end(), [&](int32_t a, int32_t c) { return area[a] > area[c]; });
    // device buffers
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) { delete b; return SA_E_CUDA; }
    for (auto *sm : b->models) {
        st = ensure_device_model(sm);
        if (st) { cudaSetDevice(prev); delete b; return st; }
    }
    const size_t nd = b->xl.size();
    st = SA_OK;
    if (!st) st = dalloc(&b->d_regions, b->regions.size());
    if (!st) st = dalloc(&b->d_order, b->order.size());
    if (!st) st = dalloc(&b->d_models, b->models.size());
    if (!st) st = dalloc(&b->d_read_scale, b->read_scale.size());
    if (!st) st = dalloc(&b->d_xl, nd);
    if (!st) st = dalloc(&b->d_xr, nd);
    if (!st) st = dalloc(&b->d_coff, nd);
    if (!st) st = dalloc(&b->d_windows, b->windows.size());
    if (!st) st = dalloc(&b->d_kmer, b->kmer.size());
    if (!st) st = dalloc(&b->d_events_raw, b->events.size());
    if (!st) st = dalloc(&b->d_events, b->events.size());
    if (!st) st = dalloc(&b->d_F, 3 * (size_t) b->cells);
    if (!st) st = dalloc(&b->d_base, nd);
    if (!st) st = dalloc(&b->d_fmax, nd);
    if (!st) st = dalloc(&b->d_out, (size_t) b->out_total);
    if (!st) st = dalloc(&b->d_out_count, b->regions.size());
    if (!st) st = dalloc(&b->d_loglik, b->regions.size());
    if (!st) st = dalloc(&b->d_status, (size_t) n_reads);
    if (!st) st = dalloc(&b->d_queue, 1);
    cudaSetDevice(prev);
    if (st) {
        free_batch_device(b);
        delete b;
        return st;
    }
    *out = b;
    return SA_OK;
}

sa_status sa_batch_upload(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    std::vector<ModelDesc> md(b->models.size());
    for (size_t i = 0; i < b->models.size(); ++i) {
        const sa_state_machine *sm = b->models[i];
        ModelDesc &m = md[i];
        std::memset(&m, 0, sizeof(m));
        m.kc = sm->dev.kc32;
        m.gapx = sm->dev.gapx32;
        m.emission = sm->emission;
        for (int j = 0; j < 9; ++j) m.t[j] = (float) sm->t[j];
        if (sm->emission == SA_EMIT_HDP) {
            const HdpTables &h = sm->hdp;
            m.hdp.knots = sm->dev.hdp_knots32;
            m.hdp.kmer_row = sm->dev.hdp_row32;
            m.hdp.x0 = (float) h.grid[0];
            m.hdp.dx = (float) (h.grid[1] - h.grid[0]);
            m.hdp.inv_dx = (float) (1.0 / (h.grid[1] - h.grid[0]));
            m.hdp.x_last = (float) h.grid[h.grid_length - 1];
            m.hdp.grid_length = (int32_t) h.grid_length;
        }
    }
    sa_status st = SA_OK;
    if (!st) st = h2d(b->d_regions, b->regions, s);
    if (!st) st = h2d(b->d_order, b->order, s);
    if (!st) st = h2d(b->d_models, md, s);
    if (!st) st = h2d(b->d_read_scale, b->read_scale, s);
    if (!st) st = h2d(b->d_xl, b->xl, s);
    if (!st) st = h2d(b->d_xr, b->xr, s);
    if (!st) st = h2d(b->d_coff, b->coff, s);
    if (!st) st = h2d(b->d_windows, b->windows, s);
    if (!st) st = h2d(b->d_kmer, b->kmer, s);
    if (!st) st = h2d(b->d_events_raw, b->events, s);
    if (!st && !b->events.empty()) {
        const int64_t n = (int64_t) b->events.size();
        prep_events<<<(unsigned) std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(b->d_events_raw, b->d_events, n);
        count_launch();
        if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
    }
    cudaSetDevice(prev);
    b->downloaded = false;
    return st;
}

sa_status sa_batch_run(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    sa_status st = SA_OK;
    if (cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_status, 0, sizeof(int32_t) * std::max<int64_t>(1, b->n_reads), s) != cudaSuccess ||
        cudaMemsetAsync(b->d_out_count, 0, sizeof(int64_t) * std::max<size_t>(1, b->regions.size()), s) != cudaSuccess)
        st = SA_E_CUDA;
    if (!st && !b->regions.empty()) {
        Args a;
        std::memset(&a, 0, sizeof(a));
        a.regions = b->d_regions;
        a.order = b->d_order;
        a.n_regions = (int64_t) b->regions.size();
        a.models = b->d_models;
        a.read_scale = b->d_read_scale;
        a.xl = b->d_xl;
        a.xr = b->d_xr;
        a.coff = b->d_coff;
        a.windows = b->d_windows;
        a.kmer = b->d_kmer;
        a.events = b->d_events;
        a.F = b->d_F;
        a.base = b->d_base;
        a.fmax = b->d_fmax;
        a.out = b->d_out;
        a.out_count = b->d_out_count;
        a.loglik = b->d_loglik;
        a.status = b->d_status;
        a.queue = b->d_queue;
        a.threshold = b->threshold;
        const int cpt = (b->max_width + kThreads - 1) / kThreads;
        a.cpt = std::max(1, cpt);
        const int wmax = a.cpt * kThreads;
        const size_t smem = sizeof(Shared) + sizeof(float) * (size_t) (9 * wmax * 2 + 2 * wmax);
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
        if (smem > 48 * 1024) cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, kThreads, smem);
        int64_t grid = (int64_t) std::max(1, sms) * std::max(1, per_sm);
        grid = std::min<int64_t>(grid, (int64_t) b->regions.size());
        batch_kernel<<<(unsigned) grid, kThreads, smem, s>>>(a, wmax);
        count_launch();
        if (cudaGetLastError() != cudaSuccess) st = SA_E_CUDA;
    }
    cudaSetDevice(prev);
    b->downloaded = false;
    return st;
}

sa_status sa_batch_download(sa_batch *b, void *stream) {
    if (!b) return SA_E_ARG;
    cudaStream_t s = (cudaStream_t) stream;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(b->device) != cudaSuccess) return SA_E_CUDA;
    const size_t nr = b->regions.size();
    b->out_count.assign(nr, 0);
    b->loglik.assign(nr, 0.0);
    b->dev_status.assign(b->n_reads, 0);
    sa_status st = SA_OK;
    if (nr) {
        if (cudaMemcpyAsync(b->out_count.data(), b->d_out_count, nr * sizeof(int64_t), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(b->loglik.data(), b->d_loglik, nr * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            st = SA_E_CUDA;
    }
    if (!st && b->n_reads &&
        cudaMemcpyAsync(b->dev_status.data(), b->d_status, b->n_reads * sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess)
        st = SA_E_CUDA;
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    // pairs: one copy per region segment in use
    b->read_pairs.assign(b->n_reads, {});
    b->read_ll.assign(b->n_reads, 0.0);
    for (int64_t r = 0; r < b->n_reads && !st; ++r) {
        int64_t total = 0;
        for (int64_t i = 0; i < b->read_n_regions[r]; ++i) {
            const int64_t ri = b->read_first_region[r] + i;
            total += std::min(b->out_count[ri], b->regions[ri].out_cap);
        }
        b->read_pairs[r].resize(total);
        int64_t at = 0;
        for (int64_t i = 0; i < b->read_n_regions[r]; ++i) {
            const int64_t ri = b->read_first_region[r] + i;
            const int64_t cnt = std::min(b->out_count[ri], b->regions[ri].out_cap);
            if (cnt > 0 && cudaMemcpyAsync(b->read_pairs[r].data() + at, b->d_out + b->regions[ri].out_base,
                                           cnt * sizeof(sa_aligned_pair), cudaMemcpyDeviceToHost, s) != cudaSuccess) {
                st = SA_E_CUDA;
                break;
            }
            at += cnt;
            b->read_ll[r] += b->loglik[ri];
        }
    }
    if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = SA_E_CUDA;
    cudaSetDevice(prev);
    b->downloaded = st == SA_OK;
    return st;
}

sa_status sa_align_batch(const sa_read *reads, int64_t n_reads, const sa_params *p, void *stream, sa_batch **out) {
    sa_status st = sa_batch_create(reads, n_reads, p, out);
    if (st) return st;
    st = sa_batch_upload(*out, stream);
    if (!st) st = sa_batch_run(*out, stream);
    if (!st) st = sa_batch_download(*out, stream);
    return st;
}

sa_status sa_batch_read_status(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads) return SA_E_ARG;
    if (b->read_status[read]) return (sa_status) b->read_status[read];
    if (!b->downloaded) return SA_E_ARG;
    return (sa_status) b->dev_status[read];
}

int64_t sa_batch_pair_count(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return -1;
    return (int64_t) b->read_pairs[read].size();
}

const sa_aligned_pair *sa_batch_pairs(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return nullptr;
    return b->read_pairs[read].data();
}

double sa_batch_log_likelihood(const sa_batch *b, int64_t read) {
    if (!b || read < 0 || read >= b->n_reads || !b->downloaded) return 0.0;
    return b->read_ll[read];
}

int64_t sa_batch_cells(const sa_batch *b) { return b ? b->cells : 0; }

sa_status sa_batch_transfer_bytes(const sa_batch *b, int64_t *h2d, int64_t *d2h) {
    if (!b || !h2d || !d2h) return SA_E_ARG;
    auto bytes = [](const auto &v) { return (int64_t) (v.size() * sizeof(v[0])); };
    *h2d = bytes(b->regions) + bytes(b->order) + (int64_t) (b->models.size() * sizeof(ModelDesc)) +
           bytes(b->read_scale) + bytes(b->xl) + bytes(b->xr) + bytes(b->coff) + bytes(b->windows) + bytes(b->kmer) +
           bytes(b->events);
    int64_t pairs = 0;
    for (const auto &rp : b->read_pairs) pairs += (int64_t) rp.size();
    *d2h = (int64_t) (b->regions.size() * (sizeof(int64_t) + sizeof(double))) + b->n_reads * (int64_t) sizeof(int32_t) +
           pairs * (int64_t) sizeof(sa_aligned_pair);
    return SA_OK;
}

sa_status sa_measure_fp32_peak(int32_t device, double *tflops) {
    if (!tflops) return SA_E_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return SA_E_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(float)) != cudaSuccess) { cudaSetDevice(prev); return SA_E_NOMEM; }
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        fma_probe<<<blocks, threads>>>(sink, iters, 1.0f + rep);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    count_launch(4);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    const sa_status st = cudaGetLastError() == cudaSuccess ? SA_OK : SA_E_CUDA;
    cudaSetDevice(prev);
    *tflops = 2.0 * 8.0 * (double) iters * blocks * threads / (best * 1e-3) / 1e12;
    return st;
}

int64_t sa_batch_regions(const sa_batch *b) { return b ? (int64_t) b->regions.size() : 0; }

void sa_batch_destroy(sa_batch *b) {
    if (!b) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    free_batch_device(b);
    cudaSetDevice(prev);
    delete b;
}

}  // extern "C"
