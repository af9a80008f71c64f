// Posterior and significance selection, one CTA per particle
// (convertSquaredDifferencesToWeights, src/map2d_optimizer.cpp:1077-1224;
// findAllSignificantPoints, :1226-1311; the 3D versions are
// src/map3d_optimizer.cpp:1610-1931).
//
// The reference sorts all positive weights and walks from the largest,
// summing in FP64 until the running sum exceeds f * sum (f =
// adaptive_fraction).  Only weights w >= t0 = (1 - f) * sum / X can ever be
// walked: the X hypotheses below t0 hold less than (1 - f) * sum, so the
// weights at or above t0 already exceed f * sum.  The CTA therefore keeps
// just those candidates (with their hypothesis index), sorts them in shared
// memory and walks them sequentially, reproducing the reference's FP64
// accumulation order exactly.  t0 carries a relative margin of 1e-6 of
// (1 - f) * sum, far above the rounding of the running sum; if the walk ever
// ran out of candidates, or there are more than SEL2_CAP of them, the
// particle is finished by select_fallback2_kernel in global memory.
//
// The same kernel emits the significant hypotheses (w >= significant
// weight) as the particle's contiguous segment of the SigEntry list used by
// updateOtherParams and backProjection.  Rows with more candidates than the
// shared-memory buffer holds take the exact radix select
// (select_radix_kernel) and, where a decision falls within rounding, the
// exact sort (select_fallback2_kernel); the 3D cross-correlation mode keeps
// the best hypothesis alone (cc_select_kernel).
#pragma once

#include <cstdint>

#include "estep_kernels.cuh"

namespace rome {
// internal linkage: every translation unit that launches these kernels gets its own copy
namespace {

constexpr int SEL2_THREADS = 512;
constexpr int SEL2_CAP = 8192;

// part[i*8]:  0 min_diff2, 1 sum_weight, 2 significant_weight, 3 threshold f*sum,
//             4 max weight, 5 diff2 cut for weights >= significant_weight, 6 t0, 7 diff2 cut for t0
// parti[i*8]: 0 best hypothesis, 1 nr walked, 2 overflow, 3 list count, 4 list base
__device__ __forceinline__ void bitonic_desc_kv(double* key, int* val, int n) {
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    bool desc = (i & k) == 0;
                    double x = key[i], y = key[ixj];
                    if (desc ? (x < y) : (x > y)) {
                        key[i] = y;
                        key[ixj] = x;
                        int t = val[i];
                        val[i] = val[ixj];
                        val[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(SEL2_THREADS)
    post_select2_kernel(int mode, long Xrow, PostLayout L, const float* __restrict__ diff2,
                        const double* __restrict__ pdir, const double* __restrict__ poff, double frac,
                        double* __restrict__ part, int* __restrict__ parti, const double* __restrict__ wgiven,
                        double* __restrict__ wout, SigEntry* __restrict__ list, int* __restrict__ counter, int cap,
                        int* __restrict__ seg, const unsigned* __restrict__ rowmin) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* key = (double*)smem_raw;           // SEL2_CAP
    int* idx = (int*)(key + SEL2_CAP);         // SEL2_CAP
    __shared__ double red[32];
    __shared__ float redf[32];
    __shared__ double smax[32];
    __shared__ long slo[32], se[32];
    __shared__ int ncand, s_nsig, s_over, s_m, s_base, s_cached;
    __shared__ double s_sig;
    const int i = blockIdx.x;
    // the particle's row: fixed length Xrow at i * Xrow, or (ragged rows, L.roff) its own span
    const long X = L.roff ? (long)(L.roff[i + 1] - L.roff[i]) * L.epr : Xrow;
    const long rb = L.roff ? (long)L.roff[i] * L.epr : (long)i * Xrow;
    const float* d = diff2 ? diff2 + rb : nullptr;
    const double* wg = wgiven ? wgiven + rb : nullptr;
    const double* po = poff ? poff + (long)i * L.K * L.ntr : nullptr;
    if (threadIdx.x == 0) s_cached = -1;  // set by the dense sweep when it kept the candidates

    // ---- min over computed diff2 ----
    double mn = 0.0;
    if (mode == 0 && rowmin) {
        // folded into the GEMM epilogue
        unsigned k = rowmin[i];
        mn = k == 0xFFFFFFFFu ? (double)INFINITY : (double)key_float(k);
    } else if (mode == 0) {
        float m = INFINITY;
        for (long e = threadIdx.x; e < X; e += blockDim.x) m = fminf(m, d[e]);
        for (int off = 16; off > 0; off >>= 1) m = fminf(m, __shfl_down_sync(0xffffffffu, m, off));
        if ((threadIdx.x & 31) == 0) redf[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            m = threadIdx.x < (blockDim.x >> 5) ? redf[threadIdx.x] : INFINITY;
            for (int off = 16; off > 0; off >>= 1) m = fminf(m, __shfl_down_sync(0xffffffffu, m, off));
            if (threadIdx.x == 0) redf[0] = m;
        }
        __syncthreads();
        mn = (double)redf[0];
        __syncthreads();
    }
    // ---- weights: sum, argmax (first in the reference's loop order), max prior ----
    double sum = 0.0, maxw = DBL_MIN, maxpd = 0.0;
    long best_lo = LONG_MAX, best_e = 0;
    if (mode == 0 && L.ent) {
        // ragged rows: the row order is the loop order
        for (long e = threadIdx.x; e < X; e += blockDim.x) {
            double pd, pof;
            long lo;
            if (!hyp_prior(e, i, L, pdir, po, pd, pof, lo)) continue;
            float dv = d[e];
            if (dv < INFINITY) maxpd = fmax(maxpd, pd * pof);
            double w = hyp_weight(dv, mn, pd, pof);
            if (wout) wout[rb + e] = w;
            sum += w;
            if (w > maxw || (w == maxw && w > DBL_MIN && lo < best_lo)) {
                maxw = w;
                best_lo = lo;
                best_e = e;
            }
        }
    } else if (mode == 0) {
        // dense rows [J][T]: the warp packs G = 32 / T whole orientations when T < 32 (lanes over the
        // G * T contiguous entries), else one orientation with lanes over its translations; the
        // orientation's class / direction indices advance incrementally (no division per entry).
        // Weights below 2^-60 of the smallest possible maximum weight are not summed (see skip_cut).
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
        const int J = (int)(X / L.T), nrot = L.npsi * L.nor, Kd = J / nrot;
        const int G = L.T < 32 ? 32 / L.T : 1;
        const bool active = L.T < 32 ? lane < G * L.T : true;
        const int jj = L.T < 32 ? lane / L.T : 0;
        const int t0 = L.T < 32 ? lane - jj * L.T : lane;
        const int tstep = L.T < 32 ? L.T : 32;
        // per-particle bounds of the prior pdf_orientation * pdf_offset
        double pmax = 0.0, pmin = INFINITY, omax = 0.0, omin = INFINITY;
        for (int q = threadIdx.x; q < Kd; q += blockDim.x) {
            const double v = pdir[q];
            pmax = fmax(pmax, v);
            if (v > 0.0) pmin = fmin(pmin, v);
        }
        for (int q = threadIdx.x; q < L.K * L.ntr; q += blockDim.x) {
            const double v = po[q];
            omax = fmax(omax, v);
            if (v > 0.0) omin = fmin(omin, v);
        }
        pmax = block_reduce_max(pmax, red);
        omax = block_reduce_max(omax, red);
        pmin = -block_reduce_max(-pmin, red);
        omin = -block_reduce_max(-omin, red);
        const double minpos = pmin * omin;
        // A weight pd * po * exp(-(d - mn)) with d - mn > skip_cut is below minpos * 2^-60; the entry
        // at the minimum has weight pd * po >= minpos whenever its prior is positive, so the skipped
        // weights (at most X of them) change the sum by less than X * 2^-60 of itself (~2e-13 at X =
        // 2.4e5).  The sum is checked against minpos below and recomputed in full if that premise fails.
        double skip_cut = (minpos > 0.0 && minpos < INFINITY) ? 41.6 + log(pmax * omax / minpos) : INFINITY;
        // Under the same premise (sum >= minpos) every candidate of the walk, w >= t0 = (1 - frac) * sum /
        // X (1 - 1e-6), has w >= tlow; the sweep keeps those weights with their index in the candidate
        // buffer, so that the candidate pass needs no second read of the row when they fit.  The cut of
        // the skip bound is far above (log(X / (1 - frac)) < 41.6), so no candidate is skipped.
        const double tlow0 = (skip_cut < INFINITY && frac < 1.0)
                                 ? (1.0 - frac) * minpos / (double)X * (1.0 - 1e-6) * (1.0 - 1e-9)
                                 : 0.0;
        for (int pass = 0; pass < 2; pass++) {
            sum = 0.0;
            maxw = DBL_MIN;
            maxpd = 0.0;
            best_lo = LONG_MAX;
            best_e = 0;
            const double tlow = pass == 0 ? tlow0 : 0.0;
            __syncthreads();
            if (threadIdx.x == 0) ncand = 0;
            __syncthreads();
            if (active) {
                // lane state: orientation j, its k = j / nrot (remainder rk), class c = k / ndir (remainder rc)
                int j = warp * G + jj;
                int k = j / nrot, rk = j - k * nrot;
                int c = k / L.ndir, rc = k - c * L.ndir;
                const int S = nwarp * G;
                // one entry (orientation jq of class index kq / class cq, translation t, value dv)
                auto visit = [&](int jq, int kq, int cq, int t, float dv) {
                    const long e = (long)jq * L.T + t;
                    if (!(dv < INFINITY)) {
                        if (wout) wout[rb + e] = 0.0;
                        return;
                    }
                    const int itr = L.notr == 1 ? t : t / L.notr;
                    const double pp = pdir[kq] * po[cq * L.ntr + itr];
                    maxpd = fmax(maxpd, pp);
                    const double diff = (double)dv - mn;
                    if (diff > skip_cut) return;  // written after the sweep when wout is wanted
                    if (diff > 700.) {
                        if (wout) wout[rb + e] = 0.0;
                        return;
                    }
                    const double w = pp * exp(-diff);
                    if (wout) wout[rb + e] = w;
                    sum += w;
                    if (w > 0.0 && w >= tlow) {
                        const int q = atomicAdd(&ncand, 1);
                        if (q < SEL2_CAP) {
                            key[q] = w;
                            idx[q] = (int)e;
                        }
                    }
                    if (w >= maxw && w > DBL_MIN) {
                        int kk, it2;
                        long lo;
                        decode_e(e, L, kk, it2, lo);
                        if (w > maxw || lo < best_lo) {
                            maxw = w;
                            best_lo = lo;
                            best_e = e;
                        }
                    }
                };
                auto advance = [&]() {
                    rk += S;
                    while (rk >= nrot) {
                        rk -= nrot;
                        k++;
                        if (++rc == L.ndir) {
                            rc = 0;
                            c++;
                        }
                    }
                };
                if (L.T < 32) {
                    // U loads in flight per lane before any of them is used
                    constexpr int U = 4;
                    for (; j < J; j += S * U) {
                        float dvs[U];
#pragma unroll
                        for (int u = 0; u < U; u++) {
                            const int ju = j + u * S;
                            dvs[u] = ju < J ? d[(long)ju * L.T + t0] : INFINITY;
                        }
#pragma unroll
                        for (int u = 0; u < U; u++) {
                            if (j + u * S < J) visit(j + u * S, k, c, t0, dvs[u]);
                            advance();
                        }
                    }
                } else {
                    for (; j < J; j += S) {
                        for (int t = t0; t < L.T; t += tstep) visit(j, k, c, t, d[(long)j * L.T + t]);
                        advance();
                    }
                }
            }
            if (skip_cut == INFINITY) break;
            // premise of the skip: the sum is at least the smallest positive prior
            const double tot = block_reduce_sum(sum, red);
            if (tot >= minpos * (1.0 - 1e-12)) break;
            skip_cut = INFINITY;
        }
        __syncthreads();
        // the kept weights are the candidate set's superset when they all fit and the cut held
        if (threadIdx.x == 0) s_cached = (tlow0 > 0.0 && skip_cut < INFINITY && ncand <= SEL2_CAP) ? ncand : -1;
        if (wout && skip_cut < INFINITY) {
            // skipped entries still get their (zero or negligible) weights written for the caller
            for (long e = threadIdx.x; e < X; e += blockDim.x) {
                const float dv = d[e];
                if (dv < INFINITY && (double)dv - mn > skip_cut) {
                    double pd, pof;
                    long lo;
                    hyp_prior(e, i, L, pdir, po, pd, pof, lo);
                    wout[rb + e] = hyp_weight(dv, mn, pd, pof);
                }
            }
        }
    } else {
        for (long e = threadIdx.x; e < X; e += blockDim.x) {
            double w = wg[e];
            sum += w;
            if (w > maxw || (w == maxw && w > DBL_MIN && e < best_lo)) {
                maxw = w;
                best_lo = e;
                best_e = e;
            }
        }
    }
    if (!(maxw > DBL_MIN)) {
        best_lo = LONG_MAX;
        best_e = 0;
    }
    sum = block_reduce_sum(sum, red);
    if (mode == 1) sum = part[(long)i * 8 + 1];  // the caller's exp_sum_weight
    for (int off = 16; off > 0; off >>= 1) {
        double ow = __shfl_down_sync(0xffffffffu, maxw, off);
        long olo = __shfl_down_sync(0xffffffffu, best_lo, off);
        long oe = __shfl_down_sync(0xffffffffu, best_e, off);
        if (ow > maxw || (ow == maxw && olo < best_lo)) {
            maxw = ow;
            best_lo = olo;
            best_e = oe;
        }
        maxpd = fmax(maxpd, __shfl_down_sync(0xffffffffu, maxpd, off));
    }
    if ((threadIdx.x & 31) == 0) {
        smax[threadIdx.x >> 5] = maxw;
        slo[threadIdx.x >> 5] = best_lo;
        se[threadIdx.x >> 5] = best_e;
        red[threadIdx.x >> 5] = maxpd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            if (smax[w] > smax[0] || (smax[w] == smax[0] && slo[w] < slo[0])) {
                smax[0] = smax[w];
                slo[0] = slo[w];
                se[0] = se[w];
            }
            red[0] = fmax(red[0], red[w]);
        }
        ncand = 0;
        s_over = 0;
    }
    __syncthreads();
    maxw = smax[0];
    best_e = se[0];
    maxpd = red[0];
    const double thr = frac * sum;
    const double t0 = frac < 1.0 ? (1.0 - frac) * sum / (double)X * (1.0 - 1e-6) : 0.0;
    const double dlim0 = (mode == 0 && t0 > 0.0 && maxpd > 0.0) ? mn + log(maxpd / t0) + 1e-6 * (1.0 + fabs(mn))
                                                                : INFINITY;
    __syncthreads();
    const int cached = s_cached;
    // ---- candidates w >= t0 ----
    auto candidate = [&](long e, double w) {
        if (w > 0.0 && w >= t0) {
            int q = atomicAdd(&ncand, 1);
            if (q < SEL2_CAP) {
                key[q] = w;
                idx[q] = (int)e;
            }
        }
    };
    auto diff2_candidate = [&](long e, float dv) {
        if (!(dv < INFINITY) || (double)dv > dlim0) return;
        double pd, pof;
        long lo;
        if (!hyp_prior(e, i, L, pdir, po, pd, pof, lo)) return;
        candidate(e, hyp_weight(dv, mn, pd, pof));
    };
    int sort_n = -1;  // with kept weights: the buffer's length, non-candidates marked -1
    if (cached >= 0) {
        int nc = 0;
        for (int q = threadIdx.x; q < cached; q += blockDim.x) {
            if (key[q] > 0.0 && key[q] >= t0) {
                nc++;
            } else {
                key[q] = -1.0;
                idx[q] = -1;
            }
        }
        nc = block_reduce_sum(nc, (int*)red);
        if (threadIdx.x == 0) ncand = nc;
        sort_n = cached;
    } else if (mode == 0 && (X & 3) == 0 && ((uintptr_t)d & 15) == 0) {
        // 16-byte loads, two in flight per thread
        const float4* d4 = (const float4*)d;
        const long X4 = X / 4;
        for (long q = threadIdx.x; q < X4; q += 2 * (long)blockDim.x) {
            const long q2 = q + blockDim.x;
            const float4 v0 = d4[q];
            const float4 v1 = q2 < X4 ? d4[q2] : make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
            diff2_candidate(4 * q, v0.x);
            diff2_candidate(4 * q + 1, v0.y);
            diff2_candidate(4 * q + 2, v0.z);
            diff2_candidate(4 * q + 3, v0.w);
            diff2_candidate(4 * q2, v1.x);
            diff2_candidate(4 * q2 + 1, v1.y);
            diff2_candidate(4 * q2 + 2, v1.z);
            diff2_candidate(4 * q2 + 3, v1.w);
        }
    } else {
        for (long e = threadIdx.x; e < X; e += blockDim.x) {
            if (mode == 0) diff2_candidate(e, d[e]);
            else candidate(e, wg[e]);
        }
    }
    __syncthreads();
    const int cnt = ncand;
    if (sort_n < 0) sort_n = cnt;
    if (cnt > SEL2_CAP) {
        if (threadIdx.x == 0) s_over = 1;
    } else {
        int n2 = 1;
        while (n2 < sort_n) n2 <<= 1;
        for (int q = sort_n + threadIdx.x; q < n2; q += blockDim.x) {
            key[q] = -1.0;
            idx[q] = -1;
        }
        __syncthreads();
        bitonic_desc_kv(key, idx, n2);
        if (threadIdx.x == 0) {
            double fw = 0.0, sig = 0.0;
            int ns = 0;
            bool stopped = false;
            for (int q = 0; q < cnt; q++) {
                ns++;
                sig = key[q];
                fw += sig;
                if (fw > thr) {
                    stopped = true;
                    break;
                }
            }
            // cannot happen with the margin; finish in global memory (also the
            // 3D walk into computed zero weights)
            if (!stopped && (t0 > 0.0 || L.list_zeros)) s_over = 1;
            s_sig = sig;
            s_nsig = ns;
            int m = ns;
            while (m < cnt && key[m] >= sig) m++;  // ties of the significant weight are significant too
            s_m = (ns > 0) ? m : 0;
        }
    }
    __syncthreads();
    // ---- significant list segment ----
    if (!s_over && list) {
        if (threadIdx.x == 0) {
            s_base = atomicAdd(counter, s_m);
            seg[2 * i] = s_base;
            seg[2 * i + 1] = s_m;
        }
        __syncthreads();
        const double inv = 1.0 / sum;
        (void)inv;
        for (int q = threadIdx.x; q < s_m; q += blockDim.x)
            if (s_base + q < cap) list[s_base + q] = SigEntry{i, idx[q], key[q] / sum};
    }
    if (threadIdx.x == 0) {
        double* pp = part + (long)i * 8;
        int* pi = parti + (long)i * 8;
        pp[0] = mn;
        pp[1] = sum;
        pp[2] = s_over ? 0.0 : s_sig;
        pp[3] = thr;
        pp[4] = maxw;
        pp[5] = (!s_over && s_sig > 0.0 && maxpd > 0.0) ? mn + log(maxpd / s_sig) + 1e-6 * (1.0 + fabs(mn))
                                                        : INFINITY;
        pp[6] = t0;
        pp[7] = dlim0;
        pi[0] = (int)best_e;
        pi[1] = s_over ? 0 : s_nsig;
        pi[2] = s_over;
        pi[3] = s_over ? 0 : s_m;
        pi[4] = s_over ? 0 : s_base;
    }
}

// Completes the selection of listed particles in global memory: gathers the
// candidates (w >= t0, or every positive weight when the shared-memory walk
// ran out), sorts them (bitonic, descending) and walks them.  One CTA per
// listed particle, each with its own scratch slot.
__global__ void __launch_bounds__(SEL2_THREADS)
    select_fallback2_kernel(int mode, long Xrow, PostLayout L, const float* __restrict__ diff2,
                            const double* __restrict__ pdir, const double* __restrict__ poff,
                            const double* __restrict__ wgiven, const int* __restrict__ plist, long slot_len,
                            double* __restrict__ scratch, double* __restrict__ part, int* __restrict__ parti) {
    const int i = plist[blockIdx.x];
    // the particle's row: fixed length Xrow at i * Xrow, or (ragged rows, L.roff) its own span
    const long X = L.roff ? (long)(L.roff[i + 1] - L.roff[i]) * L.epr : Xrow;
    const long rb = L.roff ? (long)L.roff[i] * L.epr : (long)i * Xrow;
    double* buf = scratch + (long)blockIdx.x * slot_len;
    __shared__ int ncand, nzero;
    __shared__ double red[32];
    double* pp = part + (long)i * 8;
    const double mn = pp[0], thr = pp[3];
    const float* d = diff2 ? diff2 + rb : nullptr;
    const double* wg = wgiven ? wgiven + rb : nullptr;
    const double* po = poff ? poff + (long)i * L.K * L.ntr : nullptr;
    if (threadIdx.x == 0) ncand = nzero = 0;
    __syncthreads();
    double maxpd = 0.0;
    for (long e = threadIdx.x; e < X; e += blockDim.x) {
        double w;
        if (mode == 0) {
            double pd, pof;
            long lo;
            if (!hyp_prior(e, i, L, pdir, po, pd, pof, lo)) continue;
            const float dv = d[e];
            if (!(dv < INFINITY)) continue;
            maxpd = fmax(maxpd, pd * pof);
            w = hyp_weight(dv, mn, pd, pof);
            if (w == 0.0 && L.list_zeros) atomicAdd(&nzero, 1);
        } else {
            w = wg[e];
        }
        if (w > 0.0) buf[atomicAdd(&ncand, 1)] = w;
    }
    for (int off = 16; off > 0; off >>= 1) maxpd = fmax(maxpd, __shfl_down_sync(0xffffffffu, maxpd, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = maxpd;
    __syncthreads();
    const int cnt = ncand;
    long n2 = 1;
    while (n2 < cnt) n2 <<= 1;
    for (long q = cnt + threadIdx.x; q < n2; q += blockDim.x) buf[q] = -1.0;
    __syncthreads();
    for (long k = 2; k <= n2; k <<= 1) {
        for (long j = k >> 1; j > 0; j >>= 1) {
            for (long q = threadIdx.x; q < n2; q += blockDim.x) {
                long ixj = q ^ j;
                if (ixj > q) {
                    bool desc = (q & k) == 0;
                    double x = buf[q], y = buf[ixj];
                    if (desc ? (x < y) : (x > y)) {
                        buf[q] = y;
                        buf[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        double fw = 0.0, sig = 0.0;
        int ns = 0;
        bool stopped = false;
        for (int q = 0; q < cnt; q++) {
            ns++;
            sig = buf[q];
            fw += sig;
            if (fw > thr) {
                stopped = true;
                break;
            }
        }
        // 3D sorts every computed weight, zeros included (map3d_optimizer.cpp:1840-1864):
        // a walk that passes all positive weights continues through the zeros
        if (!stopped && nzero > 0) {
            ns += nzero;
            sig = 0.0;
        }
        pp[2] = sig;
        parti[(long)i * 8 + 1] = ns;
        double mp = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) mp = fmax(mp, red[w]);
        pp[5] = (sig > 0.0 && mp > 0.0) ? mn + log(mp / sig) + 1e-6 * (1.0 + fabs(mn)) : INFINITY;
    }
}

// Completes the selection of listed particles without sorting every weight:
// an MSB-first radix select on the FP64 bit patterns of the positive weights
// (positive doubles order like their bits) finds the weight at which the
// descending running sum crosses f * sum, 11 bits per level: a histogram of
// counts and sums per digit, the crossing digit kept, until the crossing
// bucket holds at most SR_LEAF weights, which are sorted in shared memory and
// walked from the sum of everything above them.  The reference adds the
// weights one by one in descending order; the sums here are added in another
// order, so every comparison of the walk is checked against the rounding
// both orders can make (4 (n + 1) DBL_EPSILON S after n additions): if any
// comparison at the crossing lies within that margin the particle is marked
// in `redo` and finished by the exact sort (select_fallback2_kernel).  One
// CTA per listed particle; `scratch` holds its positive weights.
constexpr int SR_THREADS = 1024;
constexpr int SR_DIGITS = 2048;
constexpr int SR_LEAF = 2048;  // (histograms 24 KB + leaf 16 KB of static shared memory)

__global__ void __launch_bounds__(SR_THREADS)
    select_radix_kernel(int mode, long Xrow, PostLayout L, const float* __restrict__ diff2,
                        const double* __restrict__ pdir, const double* __restrict__ poff,
                        const double* __restrict__ wgiven, const int* __restrict__ plist, long slot_len,
                        double* __restrict__ scratch, double* __restrict__ part, int* __restrict__ parti,
                        int* __restrict__ redo) {
    const int i = plist[blockIdx.x];
    // the particle's row: fixed length Xrow at i * Xrow, or (ragged rows, L.roff) its own span
    const long X = L.roff ? (long)(L.roff[i + 1] - L.roff[i]) * L.epr : Xrow;
    const long rb = L.roff ? (long)L.roff[i] * L.epr : (long)i * Xrow;
    double* buf = scratch + (long)blockIdx.x * slot_len;
    __shared__ unsigned hcnt[SR_DIGITS];
    __shared__ double hsum[SR_DIGITS];
    __shared__ double leaf[SR_LEAF];
    __shared__ double red[32];
    __shared__ int ncand, nzero, nleaf;
    __shared__ int s_digit, s_leaf, s_stop;
    __shared__ double s_above;
    __shared__ long long s_above_n;
    double* pp = part + (long)i * 8;
    const double mn = pp[0], thr = pp[3];
    // only weights >= t0 = (1 - f) sum / X can be walked (post_select2_kernel's bound, diff2 cut dlim0)
    const double t0 = pp[6], dlim0 = pp[7];
    const float* d = diff2 ? diff2 + rb : nullptr;
    const double* wg = wgiven ? wgiven + rb : nullptr;
    const double* po = poff ? poff + (long)i * L.K * L.ntr : nullptr;
    if (threadIdx.x == 0) {
        ncand = nzero = nleaf = 0;
        s_above = 0.0;
        s_above_n = 0;
    }
    __syncthreads();
    // ---- the particle's positive weights (and, in 3D, the count of computed zeros) ----
    double maxpd = 0.0;
    for (long e = threadIdx.x; e < X; e += blockDim.x) {
        double w;
        if (mode == 0) {
            double pd, pof;
            long lo;
            if (!hyp_prior(e, i, L, pdir, po, pd, pof, lo)) continue;
            const float dv = d[e];
            if (!(dv < INFINITY)) continue;
            maxpd = fmax(maxpd, pd * pof);
            if (t0 > 0.0 && (double)dv > dlim0) continue;  // below t0: never walked
            w = hyp_weight(dv, mn, pd, pof);
            if (w == 0.0 && L.list_zeros) atomicAdd(&nzero, 1);
        } else {
            w = wg[e];
        }
        if (w > 0.0 && (w >= t0 || t0 <= 0.0)) buf[atomicAdd(&ncand, 1)] = w;
    }
    maxpd = block_reduce_max(maxpd, red);
    const int cnt = ncand;
    // ---- radix levels: digits of 11 bits from the top (exponent), the last one 8 bits ----
    unsigned long long prefix = 0;  // the digits fixed so far (bits above `shift + width`)
    int shift = 52, width = 11;
    bool stopped = false, leaf_ready = false;
    for (;;) {
        for (int q = threadIdx.x; q < SR_DIGITS; q += blockDim.x) {
            hcnt[q] = 0u;
            hsum[q] = 0.0;
        }
        __syncthreads();
        const unsigned long long mask = (1ull << width) - 1ull;
        // each thread adds runs of equal digits before touching shared memory: the weights of a broad
        // posterior share a few exponents, and one shared counter per digit would serialise them
        int cur = -1;
        unsigned cc = 0u;
        double cs = 0.0;
        for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
            const double w = buf[q];
            const unsigned long long k = (unsigned long long)__double_as_longlong(w);
            if ((k >> (shift + width)) != prefix) continue;
            const int dg = (int)((k >> shift) & mask);
            if (dg != cur) {
                if (cur >= 0) {
                    atomicAdd(&hcnt[cur], cc);
                    atomicAdd(&hsum[cur], cs);
                }
                cur = dg;
                cc = 0u;
                cs = 0.0;
            }
            cc++;
            cs += w;
        }
        if (cur >= 0) {
            atomicAdd(&hcnt[cur], cc);
            atomicAdd(&hsum[cur], cs);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // descending digits until the running sum crosses the threshold
            double above = s_above;
            long long an = s_above_n;
            int dg = -1;
            for (int q = (int)mask; q >= 0; q--) {
                if (hcnt[q] == 0u) continue;
                if (above + hsum[q] > thr) {
                    dg = q;
                    break;
                }
                above += hsum[q];
                an += hcnt[q];
            }
            s_digit = dg;
            // the decision every thread takes, made once here: reading hcnt after the barrier would race
            // with the threads that already clear it for the next level
            s_leaf = dg >= 0 && (hcnt[dg] <= (unsigned)SR_LEAF || shift == 0);
            s_above = above;
            s_above_n = an;
        }
        __syncthreads();
        const int dg = s_digit;
        const bool to_leaf = s_leaf != 0;
        __syncthreads();  // s_digit / s_leaf are rewritten by the next level
        if (dg < 0) break;  // the positive weights never exceed the threshold
        prefix = (prefix << width) | (unsigned long long)dg;
        if (to_leaf) {
            leaf_ready = true;
            break;
        }
        shift -= 11;
        if (shift < 0) {
            width = 11 + shift;  // the remaining low bits
            shift = 0;
        }
    }
    if (leaf_ready) {
        // the crossing bucket: every weight whose bits above `shift` match the prefix
        for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
            const double w = buf[q];
            const unsigned long long k = (unsigned long long)__double_as_longlong(w);
            if ((k >> shift) == prefix) {
                const int r = atomicAdd(&nleaf, 1);
                if (r < SR_LEAF) leaf[r] = w;
            }
        }
        __syncthreads();
        const int m = min(nleaf, SR_LEAF);  // more only when they are all equal (shift 0)
        int n2 = 1;
        while (n2 < m) n2 <<= 1;
        for (int q = m + threadIdx.x; q < n2; q += blockDim.x) leaf[q] = -1.0;
        __syncthreads();
        for (int k = 2; k <= n2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int q = threadIdx.x; q < n2; q += blockDim.x) {
                    const int o = q ^ j;
                    if (o > q) {
                        const bool desc = (q & k) == 0;
                        const double x = leaf[q], y = leaf[o];
                        if (desc ? (x < y) : (x > y)) {
                            leaf[q] = y;
                            leaf[o] = x;
                        }
                    }
                }
                __syncthreads();
            }
        if (threadIdx.x == 0) {
            double sacc = s_above, sig = 0.0;
            long long ns = s_above_n;
            bool ambiguous = false;
            const int nl = nleaf;
            // the comparison before the leaf (the sum of everything above it stays <= thr)
            if (fabs(sacc - thr) <= 4.0 * (double)(ns + 1) * DBL_EPSILON * fmax(sacc, thr)) ambiguous = true;
            for (int q = 0; q < nl; q++) {
                const double w = q < m ? leaf[q] : leaf[0];  // beyond SR_LEAF: equal weights
                sacc += w;
                ns++;
                sig = w;
                if (fabs(sacc - thr) <= 4.0 * (double)(ns + 1) * DBL_EPSILON * fmax(sacc, thr)) ambiguous = true;
                if (sacc > thr) {
                    stopped = true;
                    break;
                }
            }
            if (!stopped) ambiguous = true;  // cannot happen when the bucket crossed; leave it to the exact sort
            s_stop = ambiguous ? -1 : 1;
            if (!ambiguous) {
                pp[2] = sig;
                parti[(long)i * 8 + 1] = (int)ns;
                pp[5] = (sig > 0.0 && maxpd > 0.0) ? mn + log(maxpd / sig) + 1e-6 * (1.0 + fabs(mn)) : INFINITY;
            }
        }
    } else if (threadIdx.x == 0 && t0 > 0.0) {
        // with the t0 bound the walk must stop among the gathered weights: leave the rest to the exact sort
        s_stop = -1;
    } else if (threadIdx.x == 0) {
        // every positive weight walked without passing the threshold: the 3D walk continues through the
        // computed zeros (src/map3d_optimizer.cpp:1840-1864), which is exact whatever the order of the sum
        // only if it is clearly below the threshold
        const double sacc = s_above;
        const bool ambiguous = fabs(sacc - thr) <= 4.0 * (double)(cnt + 1) * DBL_EPSILON * fmax(sacc, thr);
        s_stop = ambiguous ? -1 : 0;
        if (!ambiguous) {
            double sig = 0.0;
            // the smallest positive weight is the last one walked
            sig = INFINITY;
            for (int q = 0; q < cnt; q++) sig = fmin(sig, buf[q]);
            if (cnt == 0) sig = 0.0;
            int ns = cnt;
            if (nzero > 0) {
                ns += nzero;
                sig = 0.0;
            }
            pp[2] = sig;
            parti[(long)i * 8 + 1] = ns;
            pp[5] = (sig > 0.0 && maxpd > 0.0) ? mn + log(maxpd / sig) + 1e-6 * (1.0 + fabs(mn)) : INFINITY;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) redo[blockIdx.x] = s_stop < 0 ? 1 : 0;
}

// list segments of listed particles (the ones the fallback finished)
__global__ void __launch_bounds__(1024)
    sig_list_some_kernel(const int* __restrict__ plist, long Xrow, PostLayout L, const float* __restrict__ diff2,
                         const double* __restrict__ pdir, const double* __restrict__ poff,
                         const double* __restrict__ part, int* __restrict__ counter, int cap,
                         SigEntry* __restrict__ list, int* __restrict__ seg) {
    const int i = plist[blockIdx.x];
    // the particle's row: fixed length Xrow at i * Xrow, or (ragged rows, L.roff) its own span
    const long X = L.roff ? (long)(L.roff[i + 1] - L.roff[i]) * L.epr : Xrow;
    const long rb = L.roff ? (long)L.roff[i] * L.epr : (long)i * Xrow;
    const double mn = part[(long)i * 8 + 0], sumw = part[(long)i * 8 + 1], sig = part[(long)i * 8 + 2];
    const double dcut = part[(long)i * 8 + 5];
    const float* d = diff2 + rb;
    const double* po = poff + (long)i * L.K * L.ntr;
    __shared__ int cnt, base;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (long e = threadIdx.x; e < X; e += blockDim.x) {
        float dv = d[e];
        double pd, pof;
        long lo;
        if (dv < INFINITY && (double)dv <= dcut && hyp_prior(e, i, L, pdir, po, pd, pof, lo)) {
            if (hyp_weight(dv, mn, pd, pof) >= sig) atomicAdd(&cnt, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        base = atomicAdd(counter, cnt);
        seg[2 * i] = base;
        seg[2 * i + 1] = cnt;
        cnt = 0;
    }
    __syncthreads();
    for (long e = threadIdx.x; e < X; e += blockDim.x) {
        float dv = d[e];
        double pd, pof;
        long lo;
        if (dv < INFINITY && (double)dv <= dcut && hyp_prior(e, i, L, pdir, po, pd, pof, lo)) {
            double w = hyp_weight(dv, mn, pd, pof);
            if (w >= sig) {
                int q = base + atomicAdd(&cnt, 1);
                if (q < cap) list[q] = SigEntry{i, (int)e, w / sumw};
            }
        }
    }
}

// exp_Mcoarse_significant from the list (pass 0: the hypothesis index is the coarse index)
__global__ void mcoarse_from_list_kernel(int n, long X, const SigEntry* __restrict__ list, char* __restrict__ mcoarse) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) mcoarse[(long)list[q].i * X + list[q].e] = 1;
}

// Cross-correlation mode (convertSquaredDifferencesToWeights with
// do_cross_correlation, src/map3d_optimizer.cpp:1626-1671): no
// marginalisation.  The computed hypothesis with the smallest diff2 (the
// largest normalised correlation; the first one in the reference's loop
// order, which is the row order, at a tie) gets weight 1 and every other
// weight is 0, so exp_sum_weight = 1, PMAX = 1, and the significance walk
// over that single listed weight (findAllSignificantPoints,
// :1812-1931) gives significant_weight = 1 and NR_SIGN = 1.  One CTA per
// particle; the part/parti layout and the list segment are those of
// post_select2_kernel.  A row with no computed hypothesis reports
// sum_weight 0 and no significant point.
__global__ void __launch_bounds__(SEL2_THREADS)
    cc_select_kernel(long Xrow, PostLayout L, const float* __restrict__ diff2, double* __restrict__ part,
                     int* __restrict__ parti, double* __restrict__ wout, SigEntry* __restrict__ list,
                     int* __restrict__ counter, int cap, int* __restrict__ seg) {
    __shared__ float sv[32];
    __shared__ long se[32];
    const int i = blockIdx.x;
    const long X = L.roff ? (long)(L.roff[i + 1] - L.roff[i]) * L.epr : Xrow;
    const long rb = L.roff ? (long)L.roff[i] * L.epr : (long)i * Xrow;
    const float* d = diff2 + rb;
    float best = INFINITY;
    long be = LONG_MAX;
    for (long e = threadIdx.x; e < X; e += blockDim.x) {
        const float v = d[e];
        if (v < best) {  // e rises within a thread: its first minimum is kept
            best = v;
            be = e;
        }
        if (wout) wout[rb + e] = 0.0;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_down_sync(0xffffffffu, best, off);
        const long oe = __shfl_down_sync(0xffffffffu, be, off);
        if (ov < best || (ov == best && oe < be)) {
            best = ov;
            be = oe;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        sv[threadIdx.x >> 5] = best;
        se[threadIdx.x >> 5] = be;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++)
            if (sv[w] < best || (sv[w] == best && se[w] < be)) {
                best = sv[w];
                be = se[w];
            }
        const bool found = best < INFINITY;
        double* pp = part + (long)i * 8;
        int* pi = parti + (long)i * 8;
        pp[0] = found ? (double)best : (double)INFINITY;
        pp[1] = found ? 1.0 : 0.0;
        pp[2] = found ? 1.0 : 0.0;
        pp[3] = 0.0;
        pp[4] = found ? 1.0 : 0.0;
        pp[5] = found ? (double)best : (double)INFINITY;
        pp[6] = 0.0;
        pp[7] = 0.0;
        int base = 0;
        if (list) {
            base = found ? atomicAdd(counter, 1) : 0;
            seg[2 * i] = base;
            seg[2 * i + 1] = found ? 1 : 0;
            if (found && base < cap) list[base] = SigEntry{i, (int)be, 1.0};
        }
        if (wout && found) wout[rb + be] = 1.0;
        pi[0] = found ? (int)be : 0;
        pi[1] = found ? 1 : 0;
        pi[2] = 0;
        pi[3] = found ? 1 : 0;
        pi[4] = base;
    }
}

struct SelectResult {
    int nlist;     // total significant entries
    int launches;  // kernels launched
};

// Posterior + selection + list for P particles.  list/seg/counter may be null
// (selection only).  Returns the list size; the caller re-runs with a larger
// capacity when it exceeds `cap` (entries past cap are not written).
inline SelectResult run_select(RomeGpuCtx* ctx, cudaStream_t st, int mode, int P, long X, PostLayout L,
                               const float* diff2, const double* pdir, const double* poff, double frac, double* part,
                               int* parti, const double* wgiven, double* wout, SigEntry* list, int* counter, int cap,
                               int* seg, const unsigned* rowmin = nullptr) {
    SelectResult res{0, 0};
    size_t smem = (sizeof(double) + sizeof(int)) * SEL2_CAP;
    ROME_CUDA(cudaFuncSetAttribute(post_select2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (counter) ROME_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
    post_select2_kernel<<<P, SEL2_THREADS, smem, st>>>(mode, X, L, diff2, pdir, poff, frac, part, parti, wgiven, wout,
                                                       list, counter, cap, seg, rowmin);
    ROME_CHECK_LAUNCH();
    res.launches++;
    std::vector<int> hpi((size_t)P * 8);
    ROME_CUDA(cudaMemcpyAsync(hpi.data(), parti, sizeof(int) * P * 8, cudaMemcpyDeviceToHost, st));
    int hcount = 0;
    if (counter) ROME_CUDA(cudaMemcpyAsync(&hcount, counter, sizeof(int), cudaMemcpyDeviceToHost, st));
    ROME_CUDA(cudaStreamSynchronize(st));
    std::vector<int> over;
    for (int i = 0; i < P; i++)
        if (hpi[(size_t)i * 8 + 2]) over.push_back(i);
    if (!over.empty()) {
        // radix select first (work proportional to the weights, not to sorting them all); the particles
        // it cannot settle exactly (a comparison within rounding of the threshold) take the exact sort
        const int slots = (int)std::min<size_t>(over.size(), 64);
        int* dli = ctx->ws[S_LIST].as<int>(2 * over.size());
        int* dredo = dli + over.size();
        stage_copy(ctx, dli, over.data(), over.size());
        {
            double* scratch = ctx->ws[S_SCRATCH].as<double>((size_t)slots * X);
            for (size_t b = 0; b < over.size(); b += slots) {
                const int nb = (int)std::min<size_t>(slots, over.size() - b);
                select_radix_kernel<<<nb, SR_THREADS, 0, st>>>(mode, X, L, diff2, pdir, poff, wgiven, dli + b, X,
                                                              scratch, part, parti, dredo + b);
                ROME_CHECK_LAUNCH();
                res.launches++;
            }
        }
        std::vector<int> hredo(over.size()), exact;
        ROME_CUDA(cudaMemcpyAsync(hredo.data(), dredo, sizeof(int) * over.size(), cudaMemcpyDeviceToHost, st));
        ROME_CUDA(cudaStreamSynchronize(st));
        for (size_t q = 0; q < over.size(); q++)
            if (hredo[q]) exact.push_back(over[q]);
        if (!exact.empty()) {
            long n2 = 1;
            while (n2 < X) n2 <<= 1;
            const int eslots = (int)std::min<size_t>(exact.size(), 64);
            double* scratch = ctx->ws[S_SCRATCH].as<double>((size_t)eslots * n2);
            int* dex = ctx->ws[S_SELEXACT].as<int>(exact.size());
            stage_copy(ctx, dex, exact.data(), exact.size());
            for (size_t b = 0; b < exact.size(); b += eslots) {
                const int nb = (int)std::min<size_t>(eslots, exact.size() - b);
                select_fallback2_kernel<<<nb, SEL2_THREADS, 0, st>>>(mode, X, L, diff2, pdir, poff, wgiven, dex + b,
                                                                    n2, scratch, part, parti);
                ROME_CHECK_LAUNCH();
                res.launches++;
            }
        }
        if (counter && mode == 0) {
            sig_list_some_kernel<<<(int)over.size(), 1024, 0, st>>>(dli, X, L, diff2, pdir, poff, part, counter, cap,
                                                                  list, seg);
            ROME_CHECK_LAUNCH();
            res.launches++;
            ROME_CUDA(cudaMemcpyAsync(&hcount, counter, sizeof(int), cudaMemcpyDeviceToHost, st));
            ROME_CUDA(cudaStreamSynchronize(st));
        }
    }
    res.nlist = hcount;
    return res;
}

// Cross-correlation mode selection for P particles (cc_select_kernel);
// returns the list size (one entry per particle with a computed hypothesis).
inline SelectResult run_select_cc(cudaStream_t st, int P, long X, PostLayout L, const float* diff2, double* part,
                                  int* parti, double* wout, SigEntry* list, int* counter, int cap, int* seg) {
    SelectResult res{0, 1};
    if (counter) ROME_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
    cc_select_kernel<<<P, SEL2_THREADS, 0, st>>>(X, L, diff2, part, parti, wout, list, counter, cap, seg);
    ROME_CHECK_LAUNCH();
    int hcount = 0;
    if (counter) ROME_CUDA(cudaMemcpyAsync(&hcount, counter, sizeof(int), cudaMemcpyDeviceToHost, st));
    ROME_CUDA(cudaStreamSynchronize(st));
    res.nlist = hcount;
    return res;
}

}  // namespace
}  // namespace rome
