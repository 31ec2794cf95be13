// cuda_host_runtime.h -- TEST INFRASTRUCTURE, included by cuda_host_shim.h.
// The CUDA runtime and driver calls of the library's host code
// (resistivemhd_gpu_b200/csrc/api.cu), answered on the CPU so that the
// whole C ABI can be built for the host and exercised by CPU tests: one
// "device" of compute capability 10.0 whose memory is host memory; work on
// a stream runs when it is enqueued (streams are in order and there is one
// thread); stream capture records it and a graph launch replays the record;
// events read the host clock; cuTensorMapEncodeTiled fills a HostMap.
#pragma once

#include <cstdlib>
#include <cstring>
#include <vector>

typedef struct CUevent_st *cudaEvent_t;
typedef struct CUgraph_st *cudaGraph_t;
typedef struct CUgraphExec_st *cudaGraphExec_t;

enum { cudaErrorStreamCaptureUnsupported = 900, cudaErrorMemoryAllocation = 2 };
enum { cudaStreamNonBlocking = 1 };
enum cudaStreamCaptureStatus { cudaStreamCaptureStatusNone = 0, cudaStreamCaptureStatusActive = 1 };
enum cudaStreamCaptureMode { cudaStreamCaptureModeGlobal = 0, cudaStreamCaptureModeThreadLocal = 1 };
enum cudaDeviceAttr { cudaDevAttrComputeCapabilityMajor = 75, cudaDevAttrComputeCapabilityMinor = 76 };
enum cudaDriverEntryPointQueryResult { cudaDriverEntryPointSuccess = 0 };
enum { cudaEnableDefault = 0 };

struct cudaDeviceProp {
    int major = 10, minor = 0, multiProcessorCount = 148;
};

inline const char *cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "host shim error"; }
inline cudaError_t cudaSetDevice(int d) { return d == 0 ? cudaSuccess : cudaErrorInvalidDevice; }
inline cudaError_t cudaGetDevice(int *d)
{
    *d = 0;
    return cudaSuccess;
}
inline cudaError_t cudaGetDeviceCount(int *n)
{
    *n = 1;
    return cudaSuccess;
}
inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int d)
{
    *p = cudaDeviceProp{};
    return d == 0 ? cudaSuccess : cudaErrorInvalidDevice;
}
inline cudaError_t cudaDeviceGetAttribute(int *v, cudaDeviceAttr a, int)
{
    *v = a == cudaDevAttrComputeCapabilityMajor ? 10 : 0;
    return cudaSuccess;
}

// Allocations are 256-byte aligned, as the device's are (the tensor maps and
// the pitched planes rely on it).
inline cudaError_t cudaMalloc(void *p, size_t n)
{
    void *q = nullptr;
    if (posix_memalign(&q, 256, n ? n : 1) != 0) return cudaErrorMemoryAllocation;
    std::memcpy(p, &q, sizeof q);
    return cudaSuccess;
}
template <class T> inline cudaError_t cudaMalloc(T **p, size_t n) { return cudaMalloc(static_cast<void *>(p), n); }
inline cudaError_t cudaMallocHost(void *p, size_t n) { return cudaMalloc(p, n); }
template <class T> inline cudaError_t cudaMallocHost(T **p, size_t n) { return cudaMalloc(static_cast<void *>(p), n); }
inline cudaError_t cudaFree(void *p)
{
    std::free(p);
    return cudaSuccess;
}
inline cudaError_t cudaFreeHost(void *p) { return cudaFree(p); }
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind)
{
    std::memcpy(d, s, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemset(void *p, int v, size_t n)
{
    std::memset(p, v, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpy2DAsync(void *d, size_t dpitch, const void *s, size_t spitch, size_t width, size_t height,
                                     cudaMemcpyKind, cudaStream_t = nullptr)
{
    auto op = [=] {
        for (size_t r = 0; r < height; ++r)
            std::memcpy(static_cast<char *>(d) + r * dpitch, static_cast<const char *>(s) + r * spitch, width);
    };
    if (!shim_record(op)) op();
    return cudaSuccess;
}

inline cudaError_t cudaStreamCreate(cudaStream_t *s)
{
    *s = reinterpret_cast<cudaStream_t>(new char);
    return cudaSuccess;
}
inline cudaError_t cudaStreamCreateWithFlags(cudaStream_t *s, unsigned) { return cudaStreamCreate(s); }
inline cudaError_t cudaStreamDestroy(cudaStream_t s)
{
    delete reinterpret_cast<char *>(s);
    return cudaSuccess;
}
inline cudaError_t cudaStreamIsCapturing(cudaStream_t, cudaStreamCaptureStatus *st)
{
    *st = g_capturing ? cudaStreamCaptureStatusActive : cudaStreamCaptureStatusNone;
    return cudaSuccess;
}

struct ShimGraph {
    std::vector<std::function<void()>> ops;
};
inline cudaError_t cudaStreamBeginCapture(cudaStream_t, cudaStreamCaptureMode)
{
    if (g_capturing) return cudaErrorStreamCaptureUnsupported;
    g_capture_ops = new std::vector<std::function<void()>>();
    g_capturing = true;
    return cudaSuccess;
}
inline cudaError_t cudaStreamEndCapture(cudaStream_t, cudaGraph_t *g)
{
    if (!g_capturing) return cudaErrorStreamCaptureUnsupported;
    auto *graph = new ShimGraph{std::move(*g_capture_ops)};
    delete g_capture_ops;
    g_capture_ops = nullptr;
    g_capturing = false;
    *g = reinterpret_cast<cudaGraph_t>(graph);
    return cudaSuccess;
}
inline cudaError_t cudaGraphInstantiate(cudaGraphExec_t *e, cudaGraph_t g, unsigned long long = 0)
{
    *e = reinterpret_cast<cudaGraphExec_t>(new ShimGraph(*reinterpret_cast<ShimGraph *>(g)));
    return cudaSuccess;
}
inline cudaError_t cudaGraphDestroy(cudaGraph_t g)
{
    delete reinterpret_cast<ShimGraph *>(g);
    return cudaSuccess;
}
inline cudaError_t cudaGraphExecDestroy(cudaGraphExec_t e)
{
    delete reinterpret_cast<ShimGraph *>(e);
    return cudaSuccess;
}
inline cudaError_t cudaGraphUpload(cudaGraphExec_t, cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaGraphLaunch(cudaGraphExec_t e, cudaStream_t)
{
    for (auto &op : reinterpret_cast<ShimGraph *>(e)->ops) op();
    return cudaSuccess;
}

inline cudaError_t cudaEventCreate(cudaEvent_t *e)
{
    *e = reinterpret_cast<cudaEvent_t>(new std::chrono::steady_clock::time_point());
    return cudaSuccess;
}
inline cudaError_t cudaEventDestroy(cudaEvent_t e)
{
    delete reinterpret_cast<std::chrono::steady_clock::time_point *>(e);
    return cudaSuccess;
}
inline cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t = nullptr)
{
    *reinterpret_cast<std::chrono::steady_clock::time_point *>(e) = std::chrono::steady_clock::now();
    return cudaSuccess;
}
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
inline cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b)
{
    const auto d = *reinterpret_cast<std::chrono::steady_clock::time_point *>(b) -
                   *reinterpret_cast<std::chrono::steady_clock::time_point *>(a);
    *ms = std::chrono::duration<float, std::milli>(d).count();
    return cudaSuccess;
}

// The driver's tensor-map encoder, as the library reaches it through
// cudaGetDriverEntryPoint.
typedef int CUresult;
enum { CUDA_SUCCESS = 0 };
typedef unsigned long long cuuint64_t;
typedef unsigned int cuuint32_t;
typedef int CUtensorMapDataType;
enum { CU_TENSOR_MAP_DATA_TYPE_FLOAT64 = 8 };
typedef int CUtensorMapInterleave;
typedef int CUtensorMapSwizzle;
typedef int CUtensorMapL2promotion;
typedef int CUtensorMapFloatOOBfill;
enum { CU_TENSOR_MAP_INTERLEAVE_NONE = 0, CU_TENSOR_MAP_SWIZZLE_NONE = 0, CU_TENSOR_MAP_L2_PROMOTION_L2_256B = 3,
       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE = 0 };
typedef CUresult (*PFN_cuTensorMapEncodeTiled_v12000)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                                      const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                                      const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                                      CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline CUresult shim_encode_tiled(CUtensorMap *map, CUtensorMapDataType, cuuint32_t rank, void *base,
                                  const cuuint64_t *dims, const cuuint64_t *strides, const cuuint32_t *box,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill)
{
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (rank != 2 && rank != 3)) return 1;
    HostMap h{static_cast<const double *>(base), {dims[0], dims[1], rank == 3 ? dims[2] : 1ull},
              {strides[0], rank == 3 ? strides[1] : 0ull}, {box[0], box[1], rank == 3 ? box[2] : 1u}, (int)rank};
    *map = CUtensorMap{};
    std::memcpy(map, &h, sizeof h);
    return CUDA_SUCCESS;
}
inline cudaError_t cudaGetDriverEntryPoint(const char *name, void **fn, int, cudaDriverEntryPointQueryResult *q)
{
    if (std::strcmp(name, "cuTensorMapEncodeTiled") != 0) return cudaErrorInvalidValue;
    *fn = reinterpret_cast<void *>(&shim_encode_tiled);
    *q = cudaDriverEntryPointSuccess;
    return cudaSuccess;
}
