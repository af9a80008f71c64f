// Shared definitions of librome_b200 (sm_100a): status handling, the device
// context behind RomeGpuCtx, and small device helpers.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rome_gpu.h"

namespace rome {

// ---------------------------------------------------------------------------
// errors: every entry point catches RomeFail and turns it into a status code
struct RomeFail {
    int code;
    std::string msg;
};

[[noreturn]] inline void fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw RomeFail{code, buf};
}

#define ROME_CUDA(call)                                                                                  \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            ::rome::fail(e_ == cudaErrorMemoryAllocation ? ROME_ERR_OOM : ROME_ERR_CUDA, "%s:%d %s: %s", \
                         __FILE__, __LINE__, #call, cudaGetErrorString(e_));                             \
    } while (0)

#define ROME_CHECK_LAUNCH() ROME_CUDA(cudaGetLastError())

#define ROME_REQUIRE(cond, ...)                             \
    do {                                                    \
        if (!(cond)) ::rome::fail(ROME_ERR_ARG, __VA_ARGS__); \
    } while (0)

// ---------------------------------------------------------------------------
// device buffers that grow on demand and are reused across calls
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void* get(size_t need) {
        if (need > bytes) {
            if (p) cudaFree(p);
            p = nullptr;
            bytes = 0;
            size_t want = need + need / 8 + 256;
            ROME_CUDA(cudaMalloc(&p, want));
            bytes = want;
        }
        return p;
    }
    template <typename T>
    T* as(size_t count) {
        return (T*)get(count * sizeof(T) > 0 ? count * sizeof(T) : 16);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

// device workspace slots used by the MAP2D pool driver
enum Slot {
    S_FIMG,       // windowed masked image [P][F] double2
    S_FNOMASK,    // nomask image * ctf * Minvsigma2 [P][F] double2
    S_CTF,        // local ctf [P][F] double
    S_MINV,       // Minvsigma2 [P][F] double
    S_ACT,        // active pixel list [Kact] int
    S_A,          // cross-term A operand (fp32 or bf16 hi/lo)
    S_B,          // cross-term B operand
    S_W2,         // norm GEMM A operand: Minvsigma2 * ctf^2 [P][Kp2] float
    S_Q,          // norm GEMM B operand: |P|^2 [J][Kp2] float
    S_NORM,       // norm term [P][J] float
    S_S,          // sum M |X_t|^2 [P*T] float
    S_PROJ,       // projections FP64 [J][Kact] double2
    S_DIFF2,      // diff2 [P][X] float
    S_ROTM,       // rotation matrices [J][4] double
    S_JVALID,     // orientation validity [J] int
    S_SHIFT,      // per-translation (xshift, yshift) [T] double2
    S_POFF,       // pdf_offset [P][K][ntr] double
    S_PDIR,       // pdf_direction [K] double
    S_PART,       // per particle scalars [P][8] double (min, sum, sig, thr, ...)
    S_PARTI,      // per particle ints [P][8]
    S_MCOARSE,    // coarse significance [P][K*npsi*ntr] char
    S_WCHK,       // optional weight checkpoint [P][X] double
    S_SCRATCH,    // selection scratch
    S_WSN,        // wsum_sigma2_noise accum [G][oriF] double
    S_WSUMK,      // class sums [8][K] double + group sums
    S_MRES,       // Mresol [F] int
    S_SIG2,       // sigma2_noise [G][oriF] double
    S_GROUP,      // group [P] int
    S_OLDOFF,     // old offsets [P] double2
    S_XI2,        // highres_Xi2 [P] double
    S_LIST,       // particle list of the selection fallback
    S_ROTSIG,     // Rot_significant [K*npsi] char
    S_PAIRS,      // 3D fine pass: (particle, coarse translation) pair flags, ids and list
    S_SELEXACT,   // particles whose significance walk needs the exact sort
    S_CCX,        // 3D cross-correlation mode: image norms of the pass [P] double
    S_PSCALE,     // 3D intensity-scale correction: scales [P], XA/AA spectra [P][2][oriF], data_vs_prior [K][oriF]
    S_ACTIDX,     // pixel -> active index [F] int
    S_TRANS,      // translations of the last pass [T] double2
    S_LISTCNT,    // list counter + per-orientation counts
    S_SEG,        // per-particle list segments [P][2]
    S_SIGLIST,    // significant hypotheses, particle order then orientation order
    S_OFFJ,       // per-orientation offsets and fill counters
    S_PHASE,      // phase table of the pass [T][F] double2
    S_W2B,        // norm operand, bf16 hi/lo planes
    S_QB,         // |P|^2, bf16 hi/lo planes
    S_PIDX,       // table index of every (translation, active pixel) [T][Kact] u16
    S_ROWMIN,     // per-particle min diff2 from the GEMM epilogue [P] u32 keys
    S_REC_FW,     // reconstruct: Fweight (decentred)
    S_REC_FNW,    // reconstruct: Fnewweight
    S_REC_FCONV,  // reconstruct: complex work array
    S_REC_REAL,   // reconstruct: real-space work array
    S_REC_SMALL,  // reconstruct: radial sums, tau2, mask sums
    S_REC_VOL,    // reconstruct: output volume
    S_REC_TAB,    // reconstruct: blob table
    S_FE,         // 3D fine pass: coarse-significant points (i, r, u, itr) [E] int4
    S_FENT,       // 3D fine pass: row-layout prior index [P][stride] int2
    S_TMP0,
    S_TMP1,
    S_TMP2,
    S_ROWS,       // particle_rows of a subset pool [P] int
    S_PROP,       // proposals of a restricted search [P][nprop] int
    S_PREP_RAW,   // image preparation: raw images of a chunk (host input)
    S_PREP_R,     // image preparation: real-space work images [chunk][n][n] double
    S_PREP_C,     // image preparation: half-plane transforms [chunk][n][n/2+1] double2
    S_PREP_NC,    // image preparation: noise spectra of a chunk, row-major over (row, image) [n][chunk][n/2+1] double2
    S_PREP_NR,    // image preparation: noise images [n][chunk][n] double
    S_PREP_PART,  // image preparation: per-particle parameters [P][12] double
    S_PREP_OUT,   // image preparation: outputs when they go to the host
    S_PREP_TAB,   // image preparation: shell tables, noise sigmas, per-image sums
    S_COUNT
};

}  // namespace rome

struct RomeGpuCtx {
    int device = 0;
    int precision = ROME_PREC_FP32;
    int deterministic = 0;
    size_t workspace_limit = 0;  // RomeGpuConfig::workspace_limit (0: automatic)
    cudaStream_t stream = nullptr;
    std::string last_error;
    // class references (projectors) and accumulated backprojectors, FP64
    int ref_dim = 0, nr_classes = 0, ori_size = 0, pad_size = 0, r_max = 0, padding = 2;
    long vox = 0;  // voxels per class (pad_z * pad * padF)
    double2* proj = nullptr;
    double2* bp_data = nullptr;
    double* bp_weight = nullptr;
    rome::DevBuf ws[rome::S_COUNT];
    // host-side staging
    std::vector<double> h_tmp;
    // page-locked arena for the small per-call uploads (tables, per-particle
    // scalars): copies from it are asynchronous and do not wait behind the
    // caller's own large transfers on other streams; reset at every entry point
    // projections of the last 2D pass-0 call and what they were made from
    // (reused by the next pool of the same iteration); bumped by set_projectors
    long proj_version = 0;
    std::string proj_key;
    char* h_arena = nullptr;
    char* d_arena = nullptr;  // the arena's device (mapped) address
    size_t h_arena_cap = 0, h_arena_used = 0;
    // shift table (cos, sin) from the host's libm, identical to the reference's
    double2* d_shift_tab = nullptr;
    // device flag raised by kernels whose bounded waits expire
    int* d_err = nullptr;
    double shift_sampling = 0;
    // per-phase device timings and launch counts (rome_gpu_get_timings)
    int profile = 0;
    double phase_ms[ROME_PHASE_COUNT] = {};
    long phase_launches[ROME_PHASE_COUNT] = {};
    double phase_flops[ROME_PHASE_COUNT] = {};
    double phase_bytes[ROME_PHASE_COUNT] = {};
    long total_launches = 0;
    // the image preparation's cuFFT plans and host-built tables (prep.cu)
    void* prep_plans = nullptr;
};

namespace rome {

// start of an entry point: the stream is idle (every entry point ends with a
// synchronize; this one also covers an earlier call that failed part-way), so
// the upload arena can be reused from its start
// releases the image preparation's cuFFT plans (prep.cu)
void prep_release(RomeGpuCtx* ctx);

inline void arena_reset(RomeGpuCtx* ctx) {
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->h_arena_used = 0;
}

// device-side copy out of the mapped host arena (16-byte body when both ends are aligned, then bytes);
// static: each translation unit has its own copy
static __global__ void arena_copy_kernel(const unsigned char* __restrict__ src, unsigned char* __restrict__ dst, size_t n) {
    const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n16 = (((uintptr_t)src | (uintptr_t)dst) & 15) ? 0 : n / 16;
    for (size_t q = t0; q < n16; q += stride) ((uint4*)dst)[q] = ((const uint4*)src)[q];
    for (size_t q = n16 * 16 + t0; q < n; q += stride) dst[q] = src[q];
}

// host -> device copy of n elements on the context's stream.  Through the
// page-locked, mapped arena when it has room: the host copies into the arena
// and a kernel copies it onward, so these small per-call uploads never wait
// behind large transfers that a caller runs on the copy engines meanwhile
// (e.g. the next pool's images); otherwise a plain cudaMemcpyAsync.
template <typename T>
void stage_copy(RomeGpuCtx* ctx, T* dst, const T* host, size_t n) {
    const size_t bytes = sizeof(T) * n, at = (ctx->h_arena_used + 255) & ~(size_t)255;
    if (!n) return;
    if (ctx->h_arena && ctx->d_arena && at + bytes <= ctx->h_arena_cap) {
        memcpy(ctx->h_arena + at, host, bytes);
        ctx->h_arena_used = at + bytes;
        const unsigned grid = (unsigned)std::min<size_t>((bytes / 16 + 255) / 256 + 1, 64);
        arena_copy_kernel<<<grid, 256, 0, ctx->stream>>>((const unsigned char*)(ctx->d_arena + at),
                                                         (unsigned char*)dst, bytes);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) fail(ROME_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
        return;
    }
    cudaError_t e = cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) fail(ROME_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
}

// run a function, converting RomeFail into a status and recording the message
template <typename F>
int guarded(RomeGpuCtx* ctx, F&& f) {
    try {
        f();
        return ROME_OK;
    } catch (const RomeFail& e) {
        if (ctx) ctx->last_error = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        if (ctx) ctx->last_error = e.what();
        return ROME_ERR_ARG;
    }
}

// Phase timer: CUDA events on the context's stream around each phase (when
// profiling is on) and launch / work counters (always).
class Profiler {
  public:
    explicit Profiler(RomeGpuCtx* c) : ctx_(c) {}
    ~Profiler() {
        for (auto& r : recs_) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
    }
    void begin(int ph) {
        if (!ctx_->profile) return;
        Rec r{ph, nullptr, nullptr};
        ROME_CUDA(cudaEventCreate(&r.a));
        ROME_CUDA(cudaEventCreate(&r.b));
        ROME_CUDA(cudaEventRecord(r.a, ctx_->stream));
        recs_.push_back(r);
    }
    void end(int ph) {
        if (!ctx_->profile) return;
        for (auto it = recs_.rbegin(); it != recs_.rend(); ++it)
            if (it->phase == ph) {
                ROME_CUDA(cudaEventRecord(it->b, ctx_->stream));
                return;
            }
    }
    void launched(int ph, int n = 1) {
        ctx_->phase_launches[ph] += n;
        ctx_->total_launches += n;
    }
    void add_flops(int ph, double f) { ctx_->phase_flops[ph] += f; }
    void add_bytes(int ph, double b) { ctx_->phase_bytes[ph] += b; }
    // call after the stream is synchronised
    void collect() {
        for (auto& r : recs_) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) ctx_->phase_ms[r.phase] += ms;
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        recs_.clear();
    }

  private:
    struct Rec {
        int phase;
        cudaEvent_t a, b;
    };
    RomeGpuCtx* ctx_;
    std::vector<Rec> recs_;
};

// round-to-nearest FP64 helpers used where the reference's operation order
// must be reproduced exactly (no fused multiply-add)
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

constexpr double kPi = 3.14159265358979323846;  // src/macros.h:69

}  // namespace rome
