// Runtime services of the C ABI: error reporting, argument checks, scratch buffers, state memory.
#include <atomic>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "qs_internal.cuh"

namespace qs {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return QS_OK;
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the sticky-free allocation error
        return set_error(QS_ERR_OUT_OF_MEMORY, msg);
    }
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return set_error(QS_ERR_NO_DEVICE, msg);
    return set_error(QS_ERR_CUDA, msg);
}

static std::atomic<unsigned long long> g_launches{0};

static thread_local bool g_capturing = false;
void set_capturing(bool on) { g_capturing = on; }
int refuse_if_capturing(const char* what) {
    if (!g_capturing) return QS_OK;
    return set_error(QS_ERR_NOT_SUPPORTED, std::string(what) + " copies its matrix from host memory at each run");
}

void count_launches(long long delta) {
    g_launches.fetch_add((unsigned long long)delta, std::memory_order_relaxed);
}

int check_launch(const char* kernel) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return check_cuda(e, kernel);
    return QS_OK;
}

int check_dim(ITYPE dim, UINT* n_out) {
    if (dim < 2 || (dim & (dim - 1)) != 0)
        return set_error(QS_ERR_INVALID_ARGUMENT, "dim must be a power of two >= 2");
    UINT n = 0;
    while ((1ULL << n) < dim) ++n;
    if (n > (UINT)kMaxQubits) return set_error(QS_ERR_NOT_SUPPORTED, "more than 40 qubits");
    *n_out = n;
    return QS_OK;
}

int check_target(UINT target, UINT n, const char* what) {
    if (target >= n)
        return set_error(QS_ERR_INVALID_ARGUMENT,
            std::string(what) + ": qubit index " + std::to_string(target) + " >= qubit count " +
                std::to_string(n));
    return QS_OK;
}

int check_distinct(const UINT* list, UINT count, UINT n, const char* what) {
    ITYPE seen = 0;
    for (UINT i = 0; i < count; ++i) {
        QS_TRY(check_target(list[i], n, what));
        if (seen & (1ULL << list[i]))
            return set_error(QS_ERR_INVALID_ARGUMENT, std::string(what) + ": duplicated qubit index");
        seen |= 1ULL << list[i];
    }
    return QS_OK;
}

struct ScratchBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};
static std::mutex g_scratch_mu;
static std::map<std::pair<int, cudaStream_t>, ScratchBuf> g_scratch;

int scratch(cudaStream_t stream, size_t bytes, void** out) {
    int dev = 0;
    QS_CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    ScratchBuf& b = g_scratch[{dev, stream}];
    if (b.bytes < bytes) {
        size_t want = bytes < (1u << 20) ? (1u << 20) : bytes;
        if (b.ptr) {
            // The previous buffer may still be read by work queued on this stream.
            QS_CUDA_CHECK(cudaStreamSynchronize(stream));
            QS_CUDA_CHECK(cudaFree(b.ptr));
            b.ptr = nullptr;
            b.bytes = 0;
        }
        QS_CUDA_CHECK(cudaMalloc(&b.ptr, want));
        b.bytes = want;
    }
    *out = b.ptr;
    return QS_OK;
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

// ---------------------------------------------------------------- kernels
__global__ void k_fill_basis_c128(double2* s, ITYPE dim, ITYPE basis) {
    ITYPE i = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (; i < dim; i += stride) st_stream(s + i, make_double2(i == basis ? 1.0 : 0.0, 0.0));
}
__global__ void k_fill_basis_c64(float2* s, ITYPE dim, ITYPE basis) {
    ITYPE i = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (; i < dim; i += stride) s[i] = make_float2(i == basis ? 1.f : 0.f, 0.f);
}
__global__ void k_to_c64(const double2* __restrict__ a, float2* __restrict__ b, ITYPE dim) {
    ITYPE i = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (; i < dim; i += stride) {
        double2 v = ld_stream(a + i);
        b[i] = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
    }
}
__global__ void k_to_c128(const float2* __restrict__ a, double2* __restrict__ b, ITYPE dim) {
    ITYPE i = (ITYPE)blockIdx.x * blockDim.x + threadIdx.x;
    const ITYPE stride = (ITYPE)gridDim.x * blockDim.x;
    for (; i < dim; i += stride) {
        float2 v = a[i];
        st_stream(b + i, make_double2((double)v.x, (double)v.y));
    }
}

static unsigned grid_for(ITYPE work, unsigned threads) {
    ITYPE blocks = (work + threads - 1) / threads;
    ITYPE cap = (ITYPE)sm_count() * 16;
    return (unsigned)(blocks < cap ? (blocks ? blocks : 1) : cap);
}

}  // namespace qs

using namespace qs;

extern "C" {

QS_API const char* qs_get_last_error(void) { return g_last_error.c_str(); }
QS_API const char* qs_version(void) { return "qulacs_b200 0.1.0 (sm_100a)"; }
QS_API unsigned long long qs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

QS_API int qs_device_synchronize(void) {
    QS_CUDA_CHECK(cudaDeviceSynchronize());
    return QS_OK;
}
QS_API int qs_stream_synchronize(void* stream) {
    QS_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return QS_OK;
}
QS_API int qs_stream_create(void** stream_out) {
    if (!stream_out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    cudaStream_t s = nullptr;
    QS_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream_out = (void*)s;
    return QS_OK;
}
QS_API int qs_stream_create_with_priority(int high, void** stream_out) {
    if (!stream_out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    int least = 0, greatest = 0;
    QS_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    cudaStream_t s = nullptr;
    QS_CUDA_CHECK(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high ? greatest : least));
    *stream_out = (void*)s;
    return QS_OK;
}
QS_API int qs_stream_destroy(void* stream) {
    if (!stream) return QS_OK;
    QS_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    {
        // this stream's scratch buffers (any device) go with it
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        for (auto it = g_scratch.begin(); it != g_scratch.end();) {
            if (it->first.second == (cudaStream_t)stream) {
                if (it->second.ptr) cudaFree(it->second.ptr);
                it = g_scratch.erase(it);
            } else {
                ++it;
            }
        }
    }
    QS_CUDA_CHECK(cudaStreamDestroy((cudaStream_t)stream));
    return QS_OK;
}

static int allocate_bytes(ITYPE dim, size_t elem, void** out) {
    if (!out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    UINT n;
    QS_TRY(check_dim(dim, &n));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(QS_ERR_NO_DEVICE, "no CUDA device");
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, (size_t)dim * elem);
    if (e != cudaSuccess) return check_cuda(e, "cudaMalloc(state)");
    *out = p;
    return QS_OK;
}

QS_API int qs_allocate_quantum_state(QS_ITYPE dim, void** state_out) {
    return allocate_bytes(dim, 16, state_out);
}
QS_API int qs_allocate_quantum_state_c64(QS_ITYPE dim, void** state_out) {
    return allocate_bytes(dim, 8, state_out);
}
QS_API int qs_allocate_bytes(QS_ITYPE bytes, void** out) {
    if (!out) return set_error(QS_ERR_INVALID_ARGUMENT, "null output pointer");
    *out = nullptr;
    if (bytes == 0) return set_error(QS_ERR_INVALID_ARGUMENT, "zero-byte allocation");
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, (size_t)bytes);
    if (e != cudaSuccess) return check_cuda(e, "cudaMalloc(bytes)");
    *out = p;
    return QS_OK;
}
QS_API int qs_release_quantum_state(void* state) {
    if (state) QS_CUDA_CHECK(cudaFree(state));
    return QS_OK;
}

QS_API int qs_set_computational_basis(QS_ITYPE basis, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    if (basis >= dim) return set_error(QS_ERR_INVALID_ARGUMENT, "basis index >= dim");
    k_fill_basis_c128<<<grid_for(dim, 256), 256, 0, (cudaStream_t)stream>>>((double2*)state, dim, basis);
    return check_launch("k_fill_basis_c128");
}
QS_API int qs_initialize_quantum_state(void* state, QS_ITYPE dim, void* stream) {
    return qs_set_computational_basis(0, state, dim, stream);
}
QS_API int qs_initialize_quantum_state_c64(void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    k_fill_basis_c64<<<grid_for(dim, 256), 256, 0, (cudaStream_t)stream>>>((float2*)state, dim, 0);
    return check_launch("k_fill_basis_c64");
}
QS_API int qs_load_state(const void* host_src, void* state, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_CUDA_CHECK(cudaMemcpyAsync(state, host_src, (size_t)dim * 16, cudaMemcpyHostToDevice,
        (cudaStream_t)stream));
    return QS_OK;
}
QS_API int qs_get_state(const void* state, void* host_dst, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    QS_CUDA_CHECK(cudaMemcpyAsync(host_dst, state, (size_t)dim * 16, cudaMemcpyDeviceToHost,
        (cudaStream_t)stream));
    QS_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return QS_OK;
}
QS_API int qs_state_to_c64(const void* a, void* b, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    k_to_c64<<<grid_for(dim, 256), 256, 0, (cudaStream_t)stream>>>((const double2*)a, (float2*)b, dim);
    return check_launch("k_to_c64");
}
QS_API int qs_state_to_c128(const void* a, void* b, QS_ITYPE dim, void* stream) {
    UINT n;
    QS_TRY(check_dim(dim, &n));
    k_to_c128<<<grid_for(dim, 256), 256, 0, (cudaStream_t)stream>>>((const float2*)a, (double2*)b, dim);
    return check_launch("k_to_c128");
}

}  // extern "C"
