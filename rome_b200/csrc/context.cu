// Context lifetime, projector upload and backprojector access (C ABI).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"

using namespace rome;

extern "C" int rome_gpu_abi_version(void) { return ROME_GPU_ABI_VERSION; }

extern "C" int rome_gpu_create(int device, const RomeGpuConfig* cfg, RomeGpuCtx** out) {
    if (!out) return ROME_ERR_ARG;
    *out = nullptr;
    RomeGpuCtx* ctx = new RomeGpuCtx();
    int rc = guarded(ctx, [&] {
        int ndev = 0;
        ROME_CUDA(cudaGetDeviceCount(&ndev));
        ROME_REQUIRE(device >= 0 && device < ndev, "device %d out of range (%d devices)", device, ndev);
        ctx->device = device;
        ROME_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        ROME_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10)
            fail(ROME_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
                 prop.minor);
        if (cfg) {
            ctx->precision = cfg->precision;
            ctx->deterministic = cfg->deterministic;
            ctx->profile = cfg->profile;
            ctx->workspace_limit = cfg->workspace_limit;
        }
        ROME_REQUIRE(ctx->precision >= ROME_PREC_FP32 && ctx->precision <= ROME_PREC_BF16X3, "bad precision %d",
                     ctx->precision);
        ROME_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        // The 5000-entry sin/cos table of shiftImageInFourierTransform
        // (src/image.h:1486-1512), evaluated with the host's libm so the
        // device reads exactly the reference's table values.
        const int nr = 5000;
        std::vector<double2> tab(nr);
        double sampling = 2 * kPi / (double)nr;
        for (int i = 0; i < nr; i++) {
            double xx = (double)i * sampling;
            tab[i] = make_double2(cos(xx), sin(xx));
        }
        ctx->shift_sampling = sampling;
        ROME_CUDA(cudaMalloc(&ctx->d_shift_tab, sizeof(double2) * nr));
        ROME_CUDA(cudaMemcpy(ctx->d_shift_tab, tab.data(), sizeof(double2) * nr, cudaMemcpyHostToDevice));
        ROME_CUDA(cudaMalloc(&ctx->d_err, sizeof(int)));
        ROME_CUDA(cudaMemset(ctx->d_err, 0, sizeof(int)));
        ctx->h_arena_cap = (size_t)16 << 20;
        ROME_CUDA(cudaHostAlloc((void**)&ctx->h_arena, ctx->h_arena_cap, cudaHostAllocMapped));
        ROME_CUDA(cudaHostGetDevicePointer((void**)&ctx->d_arena, ctx->h_arena, 0));
    });
    if (rc != ROME_OK) {
        fprintf(stderr, "rome_gpu_create: %s\n", ctx->last_error.c_str());
        rome_gpu_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return ROME_OK;
}

extern "C" int rome_gpu_destroy(RomeGpuCtx* ctx) {
    if (!ctx) return ROME_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    rome::prep_release(ctx);
    for (auto& b : ctx->ws) b.release();
    if (ctx->proj) cudaFree(ctx->proj);
    if (ctx->bp_data) cudaFree(ctx->bp_data);
    if (ctx->bp_weight) cudaFree(ctx->bp_weight);
    if (ctx->d_shift_tab) cudaFree(ctx->d_shift_tab);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->h_arena) cudaFreeHost(ctx->h_arena);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ROME_OK;
}

extern "C" const char* rome_gpu_last_error(const RomeGpuCtx* ctx) {
    if (!ctx) return "null context";
    return ctx->last_error.c_str();
}

extern "C" int rome_gpu_set_precision(RomeGpuCtx* ctx, int precision) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        ROME_REQUIRE(precision >= ROME_PREC_FP32 && precision <= ROME_PREC_BF16X3, "bad precision %d", precision);
        ctx->precision = precision;
    });
}

extern "C" int rome_gpu_invalidate_projections(RomeGpuCtx* ctx) {
    if (!ctx) return ROME_ERR_ARG;
    ctx->proj_version++;
    ctx->proj_key.clear();
    return ROME_OK;
}

extern "C" int rome_gpu_set_projectors(RomeGpuCtx* ctx, int ref_dim, int nr_classes, int ori_size, int pad_size,
                                       int r_max, int padding_factor, const double* data) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        ROME_REQUIRE(ref_dim == 2 || ref_dim == 3, "ref_dim must be 2 or 3");
        ROME_REQUIRE(nr_classes > 0 && ori_size > 0 && pad_size > 0 && r_max >= 0 && data, "bad projector args");
        ROME_REQUIRE(padding_factor == 2, "only padding_factor 2 (the map2d/map3d default) is supported");
        ROME_REQUIRE(pad_size == 2 * (padding_factor * r_max + 1) + 1,
                     "pad_size %d inconsistent with r_max %d (ProjectorBase::initialize)", pad_size, r_max);
        ROME_CUDA(cudaSetDevice(ctx->device));
        ctx->proj_version++;
        ctx->proj_key.clear();
        long padF = pad_size / 2 + 1;
        long vox = (ref_dim == 3 ? (long)pad_size : 1L) * pad_size * padF;
        if (ctx->proj) cudaFree(ctx->proj);
        if (ctx->bp_data) cudaFree(ctx->bp_data);
        if (ctx->bp_weight) cudaFree(ctx->bp_weight);
        ctx->proj = nullptr;
        ctx->bp_data = nullptr;
        ctx->bp_weight = nullptr;
        ROME_CUDA(cudaMalloc(&ctx->proj, sizeof(double2) * vox * nr_classes));
        ROME_CUDA(cudaMalloc(&ctx->bp_data, sizeof(double2) * vox * nr_classes));
        ROME_CUDA(cudaMalloc(&ctx->bp_weight, sizeof(double) * vox * nr_classes));
        ROME_CUDA(cudaMemcpyAsync(ctx->proj, data, sizeof(double2) * vox * nr_classes, cudaMemcpyHostToDevice,
                                  ctx->stream));
        ROME_CUDA(cudaMemsetAsync(ctx->bp_data, 0, sizeof(double2) * vox * nr_classes, ctx->stream));
        ROME_CUDA(cudaMemsetAsync(ctx->bp_weight, 0, sizeof(double) * vox * nr_classes, ctx->stream));
        ROME_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->ref_dim = ref_dim;
        ctx->nr_classes = nr_classes;
        ctx->ori_size = ori_size;
        ctx->pad_size = pad_size;
        ctx->r_max = r_max;
        ctx->padding = padding_factor;
        ctx->vox = vox;
    });
}

extern "C" int rome_gpu_get_backprojector(RomeGpuCtx* ctx, int iclass, double* data, double* weight) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->bp_data) fail(ROME_ERR_STATE, "no projectors/backprojectors set");
        ROME_REQUIRE(iclass >= 0 && iclass < ctx->nr_classes, "iclass %d out of range", iclass);
        ROME_CUDA(cudaSetDevice(ctx->device));
        if (data)
            ROME_CUDA(cudaMemcpyAsync(data, ctx->bp_data + (long)iclass * ctx->vox, sizeof(double2) * ctx->vox,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        if (weight)
            ROME_CUDA(cudaMemcpyAsync(weight, ctx->bp_weight + (long)iclass * ctx->vox, sizeof(double) * ctx->vox,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        ROME_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" int rome_gpu_set_backprojector(RomeGpuCtx* ctx, int iclass, const double* data, const double* weight) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->bp_data) fail(ROME_ERR_STATE, "no projectors/backprojectors set");
        ROME_REQUIRE(iclass >= 0 && iclass < ctx->nr_classes, "iclass %d out of range", iclass);
        ROME_CUDA(cudaSetDevice(ctx->device));
        if (data)
            ROME_CUDA(cudaMemcpyAsync(ctx->bp_data + (long)iclass * ctx->vox, data, sizeof(double2) * ctx->vox,
                                      cudaMemcpyHostToDevice, ctx->stream));
        if (weight)
            ROME_CUDA(cudaMemcpyAsync(ctx->bp_weight + (long)iclass * ctx->vox, weight, sizeof(double) * ctx->vox,
                                      cudaMemcpyHostToDevice, ctx->stream));
        ROME_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

namespace rome {
namespace {
__global__ void add_volume_kernel(long n, double* __restrict__ dst, const double* __restrict__ src) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        dst[q] += src[q];
}
}  // namespace
}  // namespace rome

extern "C" int rome_gpu_add_backprojectors(RomeGpuCtx* dst, RomeGpuCtx* src, int clear_src) {
    if (!dst || !src || dst == src) return ROME_ERR_ARG;
    return guarded(dst, [&] {
        if (!dst->bp_data || !src->bp_data) fail(ROME_ERR_STATE, "no projectors/backprojectors set");
        ROME_REQUIRE(dst->device == src->device, "contexts on different devices (%d, %d)", dst->device, src->device);
        ROME_REQUIRE(dst->ref_dim == src->ref_dim && dst->nr_classes == src->nr_classes && dst->vox == src->vox,
                     "back-projector shapes differ");
        ROME_CUDA(cudaSetDevice(dst->device));
        ROME_CUDA(cudaStreamSynchronize(src->stream));
        const long n2 = 2L * dst->vox * dst->nr_classes, n1 = dst->vox * dst->nr_classes;
        add_volume_kernel<<<1184, 256, 0, dst->stream>>>(n2, (double*)dst->bp_data, (const double*)src->bp_data);
        add_volume_kernel<<<1184, 256, 0, dst->stream>>>(n1, dst->bp_weight, src->bp_weight);
        ROME_CHECK_LAUNCH();
        ROME_CUDA(cudaStreamSynchronize(dst->stream));
        if (clear_src) {
            ROME_CUDA(cudaMemsetAsync(src->bp_data, 0, sizeof(double2) * n1, src->stream));
            ROME_CUDA(cudaMemsetAsync(src->bp_weight, 0, sizeof(double) * n1, src->stream));
            ROME_CUDA(cudaStreamSynchronize(src->stream));
        }
    });
}

extern "C" int rome_gpu_backprojector_size(RomeGpuCtx* ctx, size_t* doubles) {
    if (!ctx || !doubles) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->bp_data) fail(ROME_ERR_STATE, "no projectors/backprojectors set");
        *doubles = (size_t)3 * ctx->vox * ctx->nr_classes;
    });
}

extern "C" int rome_gpu_backprojector_device_copy(RomeGpuCtx* ctx, int to_library, void* dev_buf, void* stream) {
    if (!ctx || !dev_buf) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        if (!ctx->bp_data) fail(ROME_ERR_STATE, "no projectors/backprojectors set");
        ROME_CUDA(cudaSetDevice(ctx->device));
        cudaPointerAttributes at;
        ROME_CUDA(cudaPointerGetAttributes(&at, dev_buf));
        ROME_REQUIRE(at.type == cudaMemoryTypeDevice && at.device == ctx->device,
                     "dev_buf is not device memory of device %d", ctx->device);
        cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
        if (st != ctx->stream) ROME_CUDA(cudaStreamSynchronize(ctx->stream));  // the E-step's writes first
        const size_t n = (size_t)ctx->vox * ctx->nr_classes;
        double* data = (double*)dev_buf;
        double* weight = data + 2 * n;
        if (to_library) {
            ROME_CUDA(cudaMemcpyAsync(ctx->bp_data, data, sizeof(double2) * n, cudaMemcpyDeviceToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(ctx->bp_weight, weight, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        } else {
            ROME_CUDA(cudaMemcpyAsync(data, ctx->bp_data, sizeof(double2) * n, cudaMemcpyDeviceToDevice, st));
            ROME_CUDA(cudaMemcpyAsync(weight, ctx->bp_weight, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        }
        ROME_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" int rome_gpu_get_timings(RomeGpuCtx* ctx, RomeGpuTimings* out) {
    if (!ctx || !out) return ROME_ERR_ARG;
    for (int q = 0; q < ROME_PHASE_COUNT; q++) {
        out->ms[q] = ctx->phase_ms[q];
        out->launches[q] = ctx->phase_launches[q];
        out->flops[q] = ctx->phase_flops[q];
        out->bytes[q] = ctx->phase_bytes[q];
    }
    out->total_launches = ctx->total_launches;
    return ROME_OK;
}

extern "C" int rome_gpu_reset_timings(RomeGpuCtx* ctx) {
    if (!ctx) return ROME_ERR_ARG;
    for (int q = 0; q < ROME_PHASE_COUNT; q++) {
        ctx->phase_ms[q] = 0;
        ctx->phase_launches[q] = 0;
        ctx->phase_flops[q] = 0;
        ctx->phase_bytes[q] = 0;
    }
    ctx->total_launches = 0;
    return ROME_OK;
}

namespace rome {
namespace {
// grid-stride 16-byte copy; each thread keeps four loads in flight (host reads over PCIe are latency-bound)
__global__ void __launch_bounds__(512) copy_from_host_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst,
                                                             size_t n16) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; q + 3 * stride < n16; q += 4 * stride) {
        const uint4 a = src[q], b = src[q + stride], c = src[q + 2 * stride], d = src[q + 3 * stride];
        dst[q] = a;
        dst[q + stride] = b;
        dst[q + 2 * stride] = c;
        dst[q + 3 * stride] = d;
    }
    for (; q < n16; q += stride) dst[q] = src[q];
}
}  // namespace
}  // namespace rome

extern "C" int rome_gpu_copy_from_host(RomeGpuCtx* ctx, void* dst, const void* host, size_t bytes, void* stream) {
    if (!ctx) return ROME_ERR_ARG;
    return guarded(ctx, [&] {
        ROME_REQUIRE(dst && host && ((uintptr_t)dst & 15) == 0 && ((uintptr_t)host & 15) == 0 && bytes % 16 == 0,
                     "copy_from_host: buffers must be 16-byte aligned and the size a multiple of 16");
        cudaPointerAttributes a{};
        ROME_CUDA(cudaPointerGetAttributes(&a, host));
        ROME_REQUIRE(a.type == cudaMemoryTypeHost && a.devicePointer != nullptr,
                     "copy_from_host: the host buffer is not page-locked and mapped");
        cudaPointerAttributes b{};
        ROME_CUDA(cudaPointerGetAttributes(&b, dst));
        ROME_REQUIRE(b.type == cudaMemoryTypeDevice, "copy_from_host: dst is not device memory");
        if (bytes == 0) return;
        cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
        const size_t n16 = bytes / 16;
        const unsigned grid = (unsigned)std::min<size_t>((n16 + 511) / 512, 128);
        copy_from_host_kernel<<<grid, 512, 0, st>>>((const uint4*)a.devicePointer, (uint4*)dst, n16);
        ROME_CHECK_LAUNCH();
    });
}
