// Restricted (proposal) search of the MAP2D E-step on the tensor cores.
//
// Every particle i is compared with its own nprop proposed orientations j at
// all T translations.  The cross term of the dense contraction,
//   C[i][t][j] = sum_a Re( s_t[a] * xw_i[a] * conj(P_j[a]) ),
// (s_t: translation t's phase at active pixel a, xw_i = Minvsigma2 * ctf * X_i,
// P_j the projection) is regrouped as
//   C[(i, q)][t] = sum_a Re( s_t[a] * w_iq[a] ),  w_iq = xw_i * conj(P_j(q)),
// i.e. a GEMM whose translation operand (cos, -sin per pixel, [TN][Kp]) is
// the same for every particle and whose other operand w is one row per
// (particle, proposal).  The rows of w exist only in shared memory: eight
// producer warps form them on the CUDA cores from the gathered projection
// rows and the particle's image, in the 128-byte-swizzled K-major layout the
// UMMA descriptors expect; the translation operand arrives by TMA; one
// thread issues tcgen05.mma (M = 128 rows, N = TN >= T translations, K = 16) into
// a TMEM accumulator; the producer warps read it back with tcgen05.ld and
// write diff2 = (N - 2 C + S + Xi2) / 2 with N = sum_a w2_i |P_j|^2 formed
// alongside w.  Compared with shifting every image to every translation and
// contracting those rows (T x more operand traffic and CUDA-core FLOPs),
// the per-pair work on the CUDA cores is one complex product per pixel.
//
// Precision: ROME_PREC_BF16 rounds w and the phases to bf16 (like the dense
// BF16 contraction rounds the shifted images and projections); BF16X3 keeps
// hi and lo planes of both and issues hi*hi + hi*lo + lo*hi.
//
// Every mbarrier wait is bounded; on expiry the CTA records the timeout in
// the context's error flag, drains its TMA copies and MMAs (bounded), frees
// its TMEM and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "epilogues.cuh"
#include "restricted_tc.cuh"
#include "tc_ptx.cuh"

namespace rome {
namespace {

constexpr int RT_ROWS = 128;                   // (particle, proposal) rows per tile: UMMA M
constexpr int RT_TMAX = 256;                   // translation columns: UMMA N = TN in {32, 64, 128, 256}
constexpr int RT_PRODUCERS = 256;              // 8 producer warps: 16-byte chunk = tid % 8, rows 4 (tid / 8) + u
constexpr int RT_THREADS = RT_PRODUCERS + 64;  // + one TMA warp + one MMA warp

template <int NPLANE, int TN>
struct RtSmem {
    static constexpr int A_BYTES = RT_ROWS * BK * 2;  // 16 KB per plane
    static constexpr int B_BYTES = TN * BK * 2;       // 4 KB per plane and 32 translations
    static constexpr int STAGE_BYTES = NPLANE * (A_BYTES + B_BYTES);
    // ring depth: 4, or as many stages as fit in 200 KB (2 for 256 translations in split precision)
    static constexpr int STAGES = 200 * 1024 / STAGE_BYTES < 4 ? 200 * 1024 / STAGE_BYTES : 4;
    static constexpr int TOTAL = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
};

__device__ __forceinline__ float2 bf2_to_f2(uint32_t v) {
    return make_float2(__uint_as_float(v << 16), __uint_as_float(v & 0xFFFF0000u));
}

__device__ __forceinline__ uint32_t f2_to_bf2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

template <int NPLANE, int TN>
__global__ void __launch_bounds__(RT_THREADS, NPLANE == 1 && TN <= 64 ? 2 : 1)
    restricted_tc_kernel(const __grid_constant__ CUtensorMap mapS0, const __grid_constant__ CUtensorMap mapS1,
                         long rows, int nprop, int T, int nk, int Kp, const int* __restrict__ prop,
                         const int* __restrict__ jvalid, const float2* __restrict__ xw,
                         const float* __restrict__ w2, const __nv_bfloat16* __restrict__ B, long Jrows,
                         const float* __restrict__ S, const double* __restrict__ xi2, long Xr,
                         float* __restrict__ diff2, unsigned* __restrict__ rowmin, int* err) {
    using L = RtSmem<NPLANE, TN>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = (uint64_t*)(smem + L::STAGES * L::STAGE_BYTES);  // producer arrivals
    uint64_t* bfull = full + L::STAGES;                                // TMA bytes of the translation tile
    uint64_t* empty = bfull + L::STAGES;                               // MMAs done reading the stage
    uint64_t* done = empty + L::STAGES;                                // accumulator complete
    __shared__ float norm_row[RT_ROWS];
    __shared__ uint32_t tmem_slot;
    __shared__ int timed_out;
    volatile int* vto = &timed_out;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long m0 = (long)blockIdx.x * RT_ROWS;
    constexpr uint32_t TMEM_COLS = TN;

    if (tid == 0) {
        timed_out = 0;
        for (int s = 0; s < L::STAGES; s++) {
            mbar_init(&full[s], RT_PRODUCERS / 32);  // one arrival per producer warp
            mbar_init(&bfull[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    int issued = 0;  // translation tiles the TMA thread requested (for draining after a timeout)
    if (warp < RT_PRODUCERS / 32) {
        // ---------------- producers: w = xw * conj(P) into the swizzled A tile ----------------
        // thread -> (16-byte chunk cc of the 128-byte K-block row, rows 4 rsub + u): the eight
        // threads of a row read its 128 contiguous bytes of P, a warp four whole rows per
        // step; a thread's four rows are consecutive, so they usually share the particle
        // (its image and weights are then loaded once for all four)
        const int cc = tid & 7, rsub = tid >> 3;
        const int Kh = Kp / 2;
        constexpr int NU = RT_ROWS / (RT_PRODUCERS / 8);  // rows per thread (4)
        const uint4* b0[NU];
        const uint4* b1[NU];
        bool vrow[NU], newi[NU];
        float nacc[NU];
        const float4* xr[NU];
        const float4* wr[NU];
        int iprev = -1;
#pragma unroll
        for (int u = 0; u < NU; u++) {
            const long r = m0 + NU * rsub + u;
            vrow[u] = r < rows;
            int i = 0, j = 0;
            if (vrow[u]) {
                i = (int)(r / nprop);
                j = prop[r];
            }
            newi[u] = u == 0 || i != iprev;
            iprev = i;
            b0[u] = (const uint4*)(B + (long)j * Kp);
            b1[u] = (const uint4*)(B + (Jrows + j) * (long)Kp);
            xr[u] = (const float4*)(xw + (long)i * Kh);
            wr[u] = (const float4*)(w2 + (long)i * Kh);
            nacc[u] = 0.f;
        }
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % L::STAGES;
            // the warp leaves the loop together (one lane arrives for it below)
            const bool failed = kb >= L::STAGES && !mbar_wait(&empty[s], ((kb / L::STAGES) + 1) & 1);
            if (__any_sync(0xffffffffu, failed || *vto)) {
                *vto = 1;
                break;
            }
            uint8_t* st = smem + s * L::STAGE_BYTES;
            const int px = kb * 32 + cc * 4;  // first of the chunk's 4 complex pixels
            // all loads of the step first (rows' P chunks, then the particles' image and weights)
            uint4 hv[NU], lv[NU];
#pragma unroll
            for (int u = 0; u < NU; u++) {
                hv[u] = vrow[u] ? __ldg(b0[u] + px / 4) : make_uint4(0u, 0u, 0u, 0u);
                if (NPLANE == 2) lv[u] = vrow[u] ? __ldg(b1[u] + px / 4) : make_uint4(0u, 0u, 0u, 0u);
            }
            float4 xa = make_float4(0.f, 0.f, 0.f, 0.f), xb = xa, wv = xa;
#pragma unroll
            for (int u = 0; u < NU; u++) {
                if (newi[u]) {
                    if (vrow[u]) {
                        xa = __ldg(xr[u] + px / 2);
                        xb = __ldg(xr[u] + px / 2 + 1);
                        wv = __ldg(wr[u] + px / 4);
                    } else {
                        xa = xb = wv = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
                float2 p[4] = {bf2_to_f2(hv[u].x), bf2_to_f2(hv[u].y), bf2_to_f2(hv[u].z), bf2_to_f2(hv[u].w)};
                if (NPLANE == 2) {
                    const float2 l[4] = {bf2_to_f2(lv[u].x), bf2_to_f2(lv[u].y), bf2_to_f2(lv[u].z),
                                         bf2_to_f2(lv[u].w)};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        p[e].x += l[e].x;
                        p[e].y += l[e].y;
                    }
                }
                const float2 x[4] = {make_float2(xa.x, xa.y), make_float2(xa.z, xa.w), make_float2(xb.x, xb.y),
                                     make_float2(xb.z, xb.w)};
                const float wq[4] = {wv.x, wv.y, wv.z, wv.w};
                uint32_t hi[4], lo[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const float re = fmaf(x[e].x, p[e].x, x[e].y * p[e].y);
                    const float im = fmaf(x[e].y, p[e].x, -(x[e].x * p[e].y));
                    nacc[u] = fmaf(wq[e], fmaf(p[e].x, p[e].x, p[e].y * p[e].y), nacc[u]);
                    hi[e] = f2_to_bf2(re, im);
                    if (NPLANE == 2) {
                        const float2 hf = bf2_to_f2(hi[e]);
                        lo[e] = f2_to_bf2(re - hf.x, im - hf.y);
                    }
                }
                // row rl of the tile at rl * 128 bytes; 16-byte chunk cc stored at cc ^ (rl % 8)
                const int rl = NU * rsub + u;
                const uint32_t off = (uint32_t)rl * 128u + ((uint32_t)(cc ^ (rl & 7)) << 4);
                *(uint4*)(st + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                if (NPLANE == 2) *(uint4*)(st + L::A_BYTES + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
            }
            // every thread's tile writes are made visible to the tensor core's proxy, then the warp's
            // lanes are joined and one lane arrives for the warp
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&full[s]);
        }
        // each row's norm term: the sum over its eight chunk threads (consecutive lanes)
#pragma unroll
        for (int u = 0; u < NU; u++) {
            float v = nacc[u];
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            if (cc == 0) norm_row[NU * rsub + u] = v;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(RT_PRODUCERS) : "memory");

        // ---------------- epilogue (warps 0-3: TMEM lanes 32 w .. 32 w + 31 = rows) ----------------
        if (!mbar_wait(done, 0)) *vto = 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int bad = __shfl_sync(0xffffffffu, *vto, 0);
        if (warp < 4 && !bad) {
            const int rl = tid;  // 0..127
            const long r = m0 + rl;
            const bool valid = r < rows;
            int i = 0, j = 0;
            if (valid) {
                i = (int)(r / nprop);
                j = prop[r];
            }
            const float nrm = norm_row[rl];
            const uint32_t tb = tmem + ((uint32_t)(warp * 32) << 16);
            float m = INFINITY;
            int q = 0;
            double sx = 0.0;
            bool jv = false;
            if (valid) {
                q = (int)(r - (long)i * nprop);
                sx = (double)S[i] + xi2[i];
                jv = jvalid[j] != 0;
            }
            float* out = diff2 + (long)i * Xr + (long)q * T;
            // 32 translation columns at a time (tcgen05.ld is warp-collective: every lane takes part)
#pragma unroll 1
            for (int t0 = 0; t0 < T; t0 += 32) {
                float v[32];
                tmem_ld16(tb + t0, v);
                tmem_ld16(tb + t0 + 16, v + 16);
                if (valid) {
#pragma unroll
                    for (int u = 0; u < 32; u++) {
                        if (t0 + u < T) {
                            const float d =
                                jv ? (float)(0.5 * ((double)nrm - 2.0 * (double)v[u] + sx)) : INFINITY;
                            out[t0 + u] = d;
                            m = fminf(m, d);
                        }
                    }
                }
            }
            // minimum per particle: segmented over the warp's consecutive rows
            const int key = valid ? i : -1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float mo = __shfl_down_sync(0xffffffffu, m, o);
                const int ko = __shfl_down_sync(0xffffffffu, key, o);
                if (lane + o < 32 && ko == key) m = fminf(m, mo);
            }
            const int kprev = __shfl_up_sync(0xffffffffu, key, 1);
            if (valid && (lane == 0 || kprev != key) && m < INFINITY) atomicMin(&rowmin[i], float_key(m));
        }
    } else if (warp == RT_PRODUCERS / 32) {
        // ---------------- TMA: translation operand tiles ----------------
        if (lane == 0) {
            for (int kb = 0; kb < nk; kb++) {
                const int s = kb % L::STAGES;
                if (kb >= L::STAGES && !mbar_wait(&empty[s], ((kb / L::STAGES) + 1) & 1)) {
                    *vto = 1;
                    break;
                }
                if (*vto) break;
                uint8_t* st = smem + s * L::STAGE_BYTES + NPLANE * L::A_BYTES;
                mbar_expect_tx(&bfull[s], NPLANE * L::B_BYTES);
                tma_load_2d(st, &mapS0, &bfull[s], kb * BK, 0);
                if (NPLANE == 2) tma_load_2d(st + L::B_BYTES, &mapS1, &bfull[s], kb * BK, 0);
                issued = kb + 1;
            }
        }
    } else {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16<TN>();
            for (int kb = 0; kb < nk; kb++) {
                const int s = kb % L::STAGES;
                const uint32_t par = (kb / L::STAGES) & 1;
                if (!mbar_wait(&full[s], par) || !mbar_wait(&bfull[s], par)) {
                    *vto = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                uint8_t* st = smem + s * L::STAGE_BYTES;
                const uint32_t a0 = smem_u32(st), a1 = a0 + L::A_BYTES;
                const uint32_t b0 = smem_u32(st + NPLANE * L::A_BYTES), b1 = b0 + L::B_BYTES;
#pragma unroll
                for (int k = 0; k < BK / 16; k++) {
                    const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
                    umma_bf16(tmem, sw128_desc(a0 + 32 * k), sw128_desc(b0 + 32 * k), idesc, acc);
                    if (NPLANE == 2) {
                        umma_bf16(tmem, sw128_desc(a0 + 32 * k), sw128_desc(b1 + 32 * k), idesc, 1u);
                        umma_bf16(tmem, sw128_desc(a1 + 32 * k), sw128_desc(b0 + 32 * k), idesc, 1u);
                    }
                }
                umma_commit(&empty[s]);
            }
            // also after an early exit: `done` completes once the issued MMAs have
            umma_commit(done);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*vto) {
        if (warp == RT_PRODUCERS / 32 && lane == 0)
            for (int kb = (issued > L::STAGES ? issued - L::STAGES : 0); kb < issued; kb++)
                mbar_wait(&bfull[kb % L::STAGES], (kb / L::STAGES) & 1);
        if (tid == 0) {
            mbar_wait(done, 0);
            atomicExch(err, 1);
        }
        __syncthreads();
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

__global__ void restricted_prep_kernel(int F, int Kact, int Kh, const double2* __restrict__ Fimg,
                                       const double* __restrict__ lctf, const double* __restrict__ Minv,
                                       int apply_ctf, const int* __restrict__ act, float2* __restrict__ xw,
                                       float* __restrict__ w2, float* __restrict__ S) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    const double2* X = Fimg + (long)i * F;
    const double* M = Minv + (long)i * F;
    const double* C = lctf + (long)i * F;
    double s = 0.0;
    for (int n = threadIdx.x; n < F; n += blockDim.x) {
        const double2 v = X[n];
        s += M[n] * (v.x * v.x + v.y * v.y);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    for (int a = threadIdx.x; a < Kh; a += blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        float w = 0.f;
        if (a < Kact) {
            const int n = act[a];
            const double c = apply_ctf ? C[n] : 1.0;
            const double wd = apply_ctf ? M[n] * C[n] : M[n];
            v = make_float2((float)(wd * X[n].x), (float)(wd * X[n].y));
            w = (float)(M[n] * c * c);
        }
        xw[(long)i * Kh + a] = v;
        w2[(long)i * Kh + a] = w;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
        S[i] = (float)t;
    }
}

__global__ void restricted_shift_operand_kernel(int T, int TN, int Kact, int Kh, const unsigned short* __restrict__ pidx,
                                                const double2* __restrict__ tab, int split,
                                                __nv_bfloat162* __restrict__ hi, __nv_bfloat162* __restrict__ lo) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long)TN * Kh) return;
    const int t = (int)(q / Kh), a = (int)(q - (long)t * Kh);
    float cs = 0.f, sn = 0.f;
    if (t < T && a < Kact) {
        const unsigned short p = pidx[(long)t * Kact + a];
        if (p == 0xFFFF) {
            cs = 1.f;
        } else {
            const double2 c = tab[p & 0x7FFF];
            cs = (float)c.x;
            sn = (p & 0x8000) ? -(float)c.y : (float)c.y;
        }
    }
    const __nv_bfloat162 h = __floats2bfloat162_rn(cs, -sn);
    hi[q] = h;
    if (split) {
        const float2 hf = __bfloat1622float2(h);
        lo[q] = __floats2bfloat162_rn(cs - hf.x, -sn - hf.y);
    }
}

template <int NPLANE, int TN>
void launch_restricted(cudaStream_t st, long rows, int nprop, int T, int Kp, const int* prop, const int* jvalid,
                       const float2* xw, const float* w2, const void* B, long Jrows, const void* sh, const float* S,
                       const double* xi2, long Xr, float* diff2, unsigned* rowmin, int* derr) {
    using L = RtSmem<NPLANE, TN>;
    const __nv_bfloat16* s16 = (const __nv_bfloat16*)sh;
    CUtensorMap m0 = make_map(s16, TN, Kp, TN);
    CUtensorMap m1 = NPLANE == 2 ? make_map(s16 + (size_t)TN * Kp, TN, Kp, TN) : m0;
    auto kern = restricted_tc_kernel<NPLANE, TN>;
    ROME_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL));
    const unsigned grid = (unsigned)((rows + RT_ROWS - 1) / RT_ROWS);
    kern<<<grid, RT_THREADS, L::TOTAL, st>>>(m0, m1, rows, nprop, T, Kp / BK, Kp, prop, jvalid, xw, w2,
                                             (const __nv_bfloat16*)B, Jrows, S, xi2, Xr, diff2, rowmin, derr);
    ROME_CHECK_LAUNCH();
}

}  // namespace

void restricted_prep(cudaStream_t st, int P, int F, int Kact, int Kh, const double2* Fimg, const double* lctf,
                     const double* Minv, int apply_ctf, const int* act, float2* xw, float* w2, float* S) {
    restricted_prep_kernel<<<P, 256, 0, st>>>(F, Kact, Kh, Fimg, lctf, Minv, apply_ctf, act, xw, w2, S);
    ROME_CHECK_LAUNCH();
}

void restricted_shift_operand(cudaStream_t st, int T, int Kact, int Kp, const unsigned short* pidx,
                              const double2* tab, int precision, void* sh) {
    ROME_REQUIRE(T >= 1 && T <= RT_TMAX, "restricted search: %d translations (at most %d)", T, RT_TMAX);
    const int Kh = Kp / 2, TN = restricted_tile_tn(T);
    __nv_bfloat162* hi = (__nv_bfloat162*)sh;
    __nv_bfloat162* lo = hi + (size_t)TN * Kh;
    const long n = (long)TN * Kh;
    restricted_shift_operand_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        T, TN, Kact, Kh, pidx, tab, precision == ROME_PREC_BF16X3 ? 1 : 0, hi, lo);
    ROME_CHECK_LAUNCH();
}

void restricted_tc_diff2(cudaStream_t st, int precision, int P, int nprop, int T, int Kp, const int* prop,
                         const int* jvalid, const float2* xw, const float* w2, const void* B, long Jrows,
                         const void* sh, const float* S, const double* xi2, long Xr, float* diff2, unsigned* rowmin,
                         int* derr) {
    ROME_REQUIRE(T >= 1 && T <= RT_TMAX && Kp % BK == 0 && nprop >= 1, "restricted search: T %d, Kp %d, nprop %d",
                 T, Kp, nprop);
    const long rows = (long)P * nprop;
#define ROME_RT_LAUNCH(NP, TN)                                                                                     \
    launch_restricted<NP, TN>(st, rows, nprop, T, Kp, prop, jvalid, xw, w2, B, Jrows, sh, S, xi2, Xr, diff2, rowmin, \
                              derr)
#define ROME_RT_TILES(NP)               \
    switch (restricted_tile_tn(T)) {               \
        case 32: ROME_RT_LAUNCH(NP, 32); break;   \
        case 64: ROME_RT_LAUNCH(NP, 64); break;   \
        case 128: ROME_RT_LAUNCH(NP, 128); break; \
        default: ROME_RT_LAUNCH(NP, 256); break;  \
    }
    if (precision == ROME_PREC_BF16) {
        ROME_RT_TILES(1)
    } else if (precision == ROME_PREC_BF16X3) {
        ROME_RT_TILES(2)
    } else {
        fail(ROME_ERR_UNSUPPORTED, "precision %d has no tensor-core restricted path", precision);
    }
#undef ROME_RT_TILES
#undef ROME_RT_LAUNCH
}

}  // namespace rome
