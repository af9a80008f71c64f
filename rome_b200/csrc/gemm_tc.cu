// tcgen05 (5th-generation tensor core) contraction for the diff2 cross term:
//   C[m][n] = sum_k A[m][k] * B[n][k]      A, B bf16, K-major; C fp32 in TMEM
// with the diff2 epilogue applied straight out of TMEM.
//
// Persistent, warp-specialised kernel: one CTA per SM walks BM x BN = 128 x
// BN output tiles (cta_group::1, UMMA M = 128) in a grouped order (GROUP_M
// row tiles side by side, so the CTAs in flight share B tiles and a few A
// stripes in L2):
//   warp 0 / lane 0 : TMA producer (cp.async.bulk.tensor, 128B swizzle,
//                     STAGES-deep shared-memory ring over the k blocks of
//                     every tile, mbarrier complete_tx)
//   warp 1 / lane 0 : MMA issuer (tcgen05.mma kind::f16, 4 x K16 per 64-wide
//                     K block) into one of two TMEM accumulators (2 x BN
//                     columns); tcgen05.commit frees a ring stage and, after
//                     a tile's last k block, hands the accumulator over
//   warps 2-17      : epilogue, tcgen05.ld 32x32b (warp w reads TMEM lanes
//                     32(w%4)..+31 = rows of the tile; the four warps of a
//                     lane quarter take a quarter of the columns each), then
//                     free the accumulator, so tile i's epilogue runs while
//                     tile i+1's MMAs fill the other accumulator.
// Split precision (ROME_PREC_BF16X3) loads hi and lo planes of both operands
// and issues hi*hi + hi*lo + lo*hi into the same accumulator.
//
// Every mbarrier wait is bounded; on expiry the kernel records a timeout in a
// shared flag that every role polls, drains the copies and MMAs it issued
// (again bounded), frees its TMEM and returns, and the host reports
// ROME_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "common.cuh"
#include "gemm_tc.cuh"
#include "tc_ptx.cuh"

namespace rome {
namespace {

template <int BN, int NPLANE, int STAGES>
struct TcSmem {
    static constexpr int A_BYTES = BM * BK * 2;
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE_BYTES = NPLANE * (A_BYTES + B_BYTES);
    static constexpr int TOTAL = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
};

constexpr int kEpiWarps = 16;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int GROUP_M = 8;

// tile t of the grouped order -> (row tile, column tile)
__device__ __forceinline__ void tile_coords(int t, int ntm, int ntn, int& tm, int& tn) {
    const int per_group = GROUP_M * ntn;
    const int g = t / per_group, first = g * GROUP_M;
    const int gm = min(ntm - first, GROUP_M);
    const int r = t - g * per_group;
    tm = first + r % gm;
    tn = r / gm;
}

__device__ __forceinline__ bool flag_set(const int* f) { return *(volatile const int*)f != 0; }

// NPLANE = 1: bf16; NPLANE = 2: split precision (hi and lo planes)
template <int BN, int NPLANE, int STAGES, typename Epi>
__global__ void __launch_bounds__(kThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap mapA0, const __grid_constant__ CUtensorMap mapA1,
                   const __grid_constant__ CUtensorMap mapB0, const __grid_constant__ CUtensorMap mapB1, int M, int N,
                   int Kp, Epi epi, int* err) {
    using S = TcSmem<BN, NPLANE, STAGES>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = (uint64_t*)(smem + STAGES * S::STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;  // [2] accumulator ready for the epilogue
    uint64_t* tempty = tfull + 2;      // [2] accumulator drained by the epilogue
    uint32_t* tmem_slot = (uint32_t*)(tempty + 2);
    __shared__ int timed_out;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntm = (M + BM - 1) / BM, ntn = (N + BN - 1) / BN, ntiles = ntm * ntn;
    const int nk = Kp / BK;
    constexpr uint32_t TMEM_COLS = 2 * BN;  // two accumulators; a power of two >= 32

    if (threadIdx.x == 0) {
        timed_out = 0;
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            long it = 0, issued = 0;
            for (int t = blockIdx.x; t < ntiles && !flag_set(&timed_out); t += gridDim.x) {
                int tm, tn;
                tile_coords(t, ntm, ntn, tm, tn);
                const int m0 = tm * BM, n0 = tn * BN;
                for (int kb = 0; kb < nk; kb++, it++) {
                    const int s = (int)(it % STAGES);
                    if (it >= STAGES && !mbar_wait(&empty[s], (uint32_t)(((it / STAGES) + 1) & 1))) {
                        atomicExch(&timed_out, 1);
                        break;
                    }
                    if (flag_set(&timed_out)) break;
                    uint8_t* st = smem + s * S::STAGE_BYTES;
                    mbar_expect_tx(&full[s], S::STAGE_BYTES);
                    tma_load_2d(st, &mapA0, &full[s], kb * BK, m0);
                    tma_load_2d(st + S::A_BYTES, &mapB0, &full[s], kb * BK, n0);
                    if (NPLANE == 2) {
                        tma_load_2d(st + S::A_BYTES + S::B_BYTES, &mapA1, &full[s], kb * BK, m0);
                        tma_load_2d(st + 2 * S::A_BYTES + S::B_BYTES, &mapB1, &full[s], kb * BK, n0);
                    }
                    issued = it + 1;
                }
            }
            if (flag_set(&timed_out)) {
                // drain the copies still in flight (bounded) before the CTA leaves
                for (long q = (issued > STAGES ? issued - STAGES : 0); q < issued; q++)
                    mbar_wait(&full[q % STAGES], (uint32_t)((q / STAGES) & 1));
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            const uint32_t idesc = idesc_bf16<BN>();
            long it = 0;
            int lt = 0, committed = -1;
            for (int t = blockIdx.x; t < ntiles && !flag_set(&timed_out); t += gridDim.x, lt++) {
                const int b = lt & 1;
                if (lt >= 2 && !mbar_wait(&tempty[b], (uint32_t)(((lt >> 1) + 1) & 1))) {
                    atomicExch(&timed_out, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_base = tmem_base + (uint32_t)(b * BN);
                bool ok = true;
                for (int kb = 0; kb < nk; kb++, it++) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait(&full[s], (uint32_t)((it / STAGES) & 1))) {
                        atomicExch(&timed_out, 1);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    uint8_t* st = smem + s * S::STAGE_BYTES;
                    const uint32_t a0 = smem_u32(st), b0 = smem_u32(st + S::A_BYTES);
                    const uint32_t a1 = smem_u32(st + S::A_BYTES + S::B_BYTES);
                    const uint32_t b1 = smem_u32(st + 2 * S::A_BYTES + S::B_BYTES);
#pragma unroll
                    for (int j = 0; j < BK / 16; j++) {
                        // advance 16 bf16 (32 bytes) along K inside the swizzle atom
                        const uint32_t acc = (kb > 0 || j > 0) ? 1u : 0u;
                        umma_bf16(acc_base, sw128_desc(a0 + 32 * j), sw128_desc(b0 + 32 * j), idesc, acc);
                        if (NPLANE == 2) {
                            umma_bf16(acc_base, sw128_desc(a0 + 32 * j), sw128_desc(b1 + 32 * j), idesc, 1u);
                            umma_bf16(acc_base, sw128_desc(a1 + 32 * j), sw128_desc(b0 + 32 * j), idesc, 1u);
                        }
                    }
                    umma_commit(&empty[s]);
                }
                if (!ok) break;
                umma_commit(&tfull[b]);
                committed = lt;
            }
            if (flag_set(&timed_out) && committed >= 0) {
                // the last accumulator hand-over covers every MMA issued before it (bounded wait)
                mbar_wait(&tfull[committed & 1], (uint32_t)((committed >> 1) & 1));
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue ----------------
        const int q = warp & 3;                  // TMEM lane quarter this warp may read
        constexpr int kParts = kEpiWarps / 4;    // warps per lane quarter, each with 1/kParts of the columns
        constexpr int kCols = BN / kParts;       // a multiple of 16
        static_assert(kCols % 16 == 0, "column share of an epilogue warp");
        const int part = (warp - 2) >> 2;
        const int c_lo = part * kCols, c_hi = c_lo + kCols;
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, lt++) {
            const int b = lt & 1;
            if (flag_set(&timed_out)) break;
            if (!mbar_wait(&tfull[b], (uint32_t)((lt >> 1) & 1))) {
                atomicExch(&timed_out, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int tm, tn;
            tile_coords(t, ntm, ntn, tm, tn);
            const int row = tm * BM + q * 32 + lane, n0 = tn * BN;
            const uint32_t lane_base = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN);
            float rmin = INFINITY;
            const typename Epi::Row R = epi.row(row < M ? row : M - 1);
#pragma unroll 1
            for (int c = c_lo; c < c_hi; c += 16) {
                float v[16];
                tmem_ld16(lane_base + c, v);
                if (row < M && n0 + c < N) rmin = fminf(rmin, epi.chunk16(R, n0 + c, v, min(16, N - (n0 + c))));
            }
            if (row < M) epi.finish_row(row, rmin);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[b]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && timed_out) atomicExch(err, 1);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

int sm_count() {
    int dev = 0, n = 0;
    ROME_CUDA(cudaGetDevice(&dev));
    ROME_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n > 0 ? n : 1;
}

template <int BN, int NPLANE, int STAGES, typename Epi>
void launch(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, const Epi& epi, int* derr) {
    using S = TcSmem<BN, NPLANE, STAGES>;
    const __nv_bfloat16* Ah = (const __nv_bfloat16*)A;
    const __nv_bfloat16* Bh = (const __nv_bfloat16*)B;
    CUtensorMap a0 = make_map(Ah, M, Kp, BM);
    CUtensorMap b0 = make_map(Bh, N, Kp, BN);
    CUtensorMap a1 = NPLANE == 2 ? make_map(Ah + (size_t)M * Kp, M, Kp, BM) : a0;
    CUtensorMap b1 = NPLANE == 2 ? make_map(Bh + (size_t)N * Kp, N, Kp, BN) : b0;
    auto kern = tc_gemm_kernel<BN, NPLANE, STAGES, Epi>;
    ROME_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL));
    const long ntiles = (long)((M + BM - 1) / BM) * ((N + BN - 1) / BN);
    const int grid = (int)std::min<long>(ntiles, sm_count());
    kern<<<grid, kThreads, S::TOTAL, st>>>(a0, a1, b0, b1, M, N, Kp, epi, derr);
    ROME_CHECK_LAUNCH();
}

// ---- tile-shape autotuner -------------------------------------------------
// The tile width BN and the ring depth STAGES trade the number of CTAs (and
// so the balance of the last wave over 148 SMs) against the reuse of each
// A tile and the latency the ring hides; which wins depends on M, N and Kp.
// The first call with a given key -- epilogue kind, operand planes, device,
// N, Kp and the number of 128-row tiles rounded up to a power of two -- runs
// every candidate shape on that call's own operands, timed with CUDA events
// on the call's stream (one untimed run, then the median of three timed
// runs each), and keeps the fastest; later calls with the key launch it
// directly.  Only the table is locked: tuning runs outside the lock, and
// other host threads that meet a key while it is being tuned launch the
// default shape.  All candidates
// write identical outputs (each output element accumulates the same K blocks
// in the same order whatever the tile width, and the epilogues only store
// values and fold row minima), so the results do not depend on which
// candidate ran last.  With ROME_TC_TUNE=0 in the environment the first
// candidate of each list (the untuned default) is used; ROME_TC_SHAPE=<i>
// pins candidate i of each list (clamped to the list), e.g. to reproduce a
// choice.
template <typename Epi>
struct Cand {
    const char* name;
    void (*fn)(cudaStream_t, int, int, int, const void*, const void*, const Epi&, int*);
};

struct TuneKey {
    int kind, nplane, dev, N, Kp, mb;
    bool operator<(const TuneKey& o) const {
        return std::tie(kind, nplane, dev, N, Kp, mb) < std::tie(o.kind, o.nplane, o.dev, o.N, o.Kp, o.mb);
    }
};
struct TuneEntry {
    int choice = 0, ncand = 0;
    bool done = false;
    const char* names[4] = {};
    float ms[4] = {};
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;

bool tuning_enabled() {
    const char* e = getenv("ROME_TC_TUNE");
    return !(e && e[0] == '0');
}

// ROME_TC_SHAPE=<i>: the pinned candidate index, or -1
int pinned_shape() {
    const char* e = getenv("ROME_TC_SHAPE");
    if (!e || e[0] < '0' || e[0] > '9') return -1;
    return atoi(e);
}

template <typename Epi, int NC>
void tuned(int kind, int nplane, const Cand<Epi> (&c)[NC], cudaStream_t st, int M, int N, int Kp, const void* A,
           const void* B, const Epi& epi, int* derr) {
    static_assert(NC >= 1 && NC <= 4, "1-4 candidates");
    const int pin = pinned_shape();
    if (pin >= 0) {
        c[pin < NC ? pin : NC - 1].fn(st, M, N, Kp, A, B, epi, derr);
        return;
    }
    if (!tuning_enabled() || NC == 1) {
        c[0].fn(st, M, N, Kp, A, B, epi, derr);
        return;
    }
    int dev = 0;
    ROME_CUDA(cudaGetDevice(&dev));
    int mb = 1;
    while (mb < (M + BM - 1) / BM) mb <<= 1;
    const TuneKey key{kind, nplane, dev, N, Kp, mb};
    {
        // the lock covers the table only: a key being tuned by another host
        // thread runs the default shape meanwhile instead of waiting
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            const int q = it->second.done ? it->second.choice : 0;
            c[q].fn(st, M, N, Kp, A, B, epi, derr);
            return;
        }
        g_tune[key] = TuneEntry{};  // in progress
    }
    TuneEntry e;
    e.ncand = NC;
    constexpr int kReps = 3;
    cudaEvent_t ev[kReps + 1];
    for (auto& x : ev) ROME_CUDA(cudaEventCreate(&x));
    float best = 0.f;
    for (int q = 0; q < NC; q++) {
        e.names[q] = c[q].name;
        c[q].fn(st, M, N, Kp, A, B, epi, derr);
        ROME_CUDA(cudaEventRecord(ev[0], st));
        for (int r = 0; r < kReps; r++) {
            c[q].fn(st, M, N, Kp, A, B, epi, derr);
            ROME_CUDA(cudaEventRecord(ev[r + 1], st));
        }
        ROME_CUDA(cudaEventSynchronize(ev[kReps]));
        float t[kReps];
        for (int r = 0; r < kReps; r++) ROME_CUDA(cudaEventElapsedTime(&t[r], ev[r], ev[r + 1]));
        std::sort(t, t + kReps);
        e.ms[q] = t[kReps / 2];  // median of the timed runs
        if (q == 0 || e.ms[q] < best) {
            best = e.ms[q];
            e.choice = q;
        }
    }
    for (auto& x : ev) cudaEventDestroy(x);
    e.done = true;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = e;
}

enum { KIND_DIFF2 = 0, KIND_STORE = 1, KIND_BIAS = 2 };

template <typename Epi>
struct Shapes {
    static constexpr Cand<Epi> one[2] = {{"256x4", launch<256, 1, 4, Epi>}, {"128x6", launch<128, 1, 6, Epi>}};
    static constexpr Cand<Epi> two[2] = {{"128x3", launch<128, 2, 3, Epi>}, {"64x4", launch<64, 2, 4, Epi>}};
};

}  // namespace

void tc_diff2_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, int precision,
                   const Diff2Epi& epi, int* derr) {
    if (precision == ROME_PREC_BF16)
        tuned(KIND_DIFF2, 1, Shapes<Diff2Epi>::one, st, M, N, Kp, A, B, epi, derr);
    else if (precision == ROME_PREC_BF16X3)
        tuned(KIND_DIFF2, 2, Shapes<Diff2Epi>::two, st, M, N, Kp, A, B, epi, derr);
    else
        fail(ROME_ERR_UNSUPPORTED, "precision %d has no tensor-core path", precision);
}

void tc_store_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, float* out, int ld,
                   int* derr) {
    tuned(KIND_STORE, 2, Shapes<StoreEpi>::two, st, M, N, Kp, A, B, StoreEpi{out, ld}, derr);
}

void tc_bias_gemm(cudaStream_t st, int M, int N, int Kp, const void* A, const void* B, float* out, int ld,
                  const float* bias, int group, int* derr, bool split) {
    const BiasStoreEpi epi{out, ld, bias, group};
    if (split)
        tuned(KIND_BIAS, 2, Shapes<BiasStoreEpi>::two, st, M, N, Kp, A, B, epi, derr);
    else
        tuned(KIND_BIAS, 1, Shapes<BiasStoreEpi>::one, st, M, N, Kp, A, B, epi, derr);
}

std::string tc_tuning_report() {
    static const char* kinds[] = {"diff2", "store", "bias"};
    std::lock_guard<std::mutex> lock(g_tune_mu);
    std::string out;
    char line[256];
    for (const auto& kv : g_tune) {
        const TuneKey& k = kv.first;
        const TuneEntry& e = kv.second;
        if (!e.done) continue;
        int n = snprintf(line, sizeof line, "%s planes=%d dev=%d N=%d Kp=%d mtiles=%d choice=%s", kinds[k.kind],
                         k.nplane, k.dev, k.N, k.Kp, k.mb, e.names[e.choice]);
        for (int q = 0; q < e.ncand && n < (int)sizeof line; q++)
            n += snprintf(line + n, sizeof line - n, " %s:%.4fms", e.names[q], e.ms[q]);
        out += line;
        out += "\n";
    }
    return out;
}

// hi/lo bf16 planes of a [rows][K] fp32 matrix, zero padded to Kpad columns
__global__ void split_bf16_kernel(const float* __restrict__ in, long rows, int K, int ldin, int Kpad,
                                  __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= rows * Kpad) return;
    long r = q / Kpad;
    int k = (int)(q - r * Kpad);
    float v = k < K ? in[r * ldin + k] : 0.f;
    __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[q] = h;
    if (lo) lo[q] = __float2bfloat16_rn(v - __bfloat162float(h));
}

void split_bf16(cudaStream_t st, const float* in, long rows, int K, int ldin, int Kpad, void* out, bool with_lo) {
    __nv_bfloat16* hi = (__nv_bfloat16*)out;
    __nv_bfloat16* lo = with_lo ? hi + rows * Kpad : nullptr;
    long n = rows * Kpad;
    split_bf16_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, rows, K, ldin, Kpad, hi, lo);
    ROME_CHECK_LAUNCH();
}

// transposed split: out[c][r] = in[r][c] (hi plane [cols][rows_pad], then lo),
// rows beyond `rows` zero; 32 x 32 tiles through shared memory
__global__ void split_bf16_t_kernel(const float* __restrict__ in, int rows, int cols, int ldin, int rows_pad,
                                    __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        tile[y][threadIdx.x] = (r < rows && c < cols) ? in[(long)r * ldin + c] : 0.f;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (c < cols && r < rows_pad) {
            const float v = tile[threadIdx.x][y];
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            hi[(long)c * rows_pad + r] = h;
            lo[(long)c * rows_pad + r] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
    }
}

void split_bf16_t(cudaStream_t st, const float* in, int rows, int cols, int ldin, int rows_pad, void* out) {
    __nv_bfloat16* hi = (__nv_bfloat16*)out;
    __nv_bfloat16* lo = hi + (size_t)cols * rows_pad;
    dim3 grid((cols + 31) / 32, (rows_pad + 31) / 32);
    split_bf16_t_kernel<<<grid, dim3(32, 8), 0, st>>>(in, rows, cols, ldin, rows_pad, hi, lo);
    ROME_CHECK_LAUNCH();
}

void tc_check_error(cudaStream_t st, int* derr) {
    int h = 0;
    ROME_CUDA(cudaMemcpyAsync(&h, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
    ROME_CUDA(cudaStreamSynchronize(st));
    if (h) {
        ROME_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), st));
        fail(ROME_ERR_TIMEOUT, "tensor-core GEMM: a bounded mbarrier wait expired");
    }
}

// A wait that runs out: one thread initialises an mbarrier that nothing
// arrives on and waits for its first phase with the same bounded wait the
// tensor-core kernels use, for limit_ns of wall time; the expiry is recorded
// in the context's error flag exactly as a kernel's would be.
__global__ void wait_selftest_kernel(uint64_t limit_ns, int* err, unsigned long long* waited_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint64_t t0 = global_ns();
    const bool ok = mbar_wait_ns(&bar, 0, limit_ns);
    *waited_ns = global_ns() - t0;
    if (!ok) atomicExch(err, 1);
}

}  // namespace rome

extern "C" int rome_gpu_wait_selftest(RomeGpuCtx* ctx, double limit_seconds, double* waited_seconds) {
    if (!ctx) return ROME_ERR_ARG;
    return rome::guarded(ctx, [&] {
        ROME_REQUIRE(limit_seconds >= 1e-4 && limit_seconds <= 2.0, "limit %g s outside [1e-4, 2]", limit_seconds);
        ROME_CUDA(cudaSetDevice(ctx->device));
        unsigned long long* dw = ctx->ws[rome::S_TMP2].as<unsigned long long>(1);
        rome::wait_selftest_kernel<<<1, 32, 0, ctx->stream>>>((uint64_t)(limit_seconds * 1e9), ctx->d_err, dw);
        ROME_CHECK_LAUNCH();
        unsigned long long h = 0;
        ROME_CUDA(cudaMemcpyAsync(&h, dw, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        ROME_CUDA(cudaStreamSynchronize(ctx->stream));
        if (waited_seconds) *waited_seconds = (double)h * 1e-9;
        ctx->total_launches += 1;
        rome::tc_check_error(ctx->stream, ctx->d_err);
    });
}

extern "C" size_t rome_gpu_tuning_report(char* buf, size_t len) {
    const std::string r = rome::tc_tuning_report();
    if (buf && len) {
        const size_t n = std::min(len - 1, r.size());
        memcpy(buf, r.data(), n);
        buf[n] = '\0';
    }
    return r.size();
}
