// C-linkage entry points over the reference GPU backend's host wrappers (src/gpusim/update_ops_cuda.h,
// memory_ops.h, stat_ops.h), for bench.py's gpusim leg (ctypes).  Used for measurement only: the library
// never links or loads this.  The host wrappers take `stream` as a pointer to a stream handle and
// dereference it, so the shim holds one stream made by the backend's own allocate_cuda_stream_host.
#include "memory_ops.h"
#include "stat_ops.h"
#include "update_ops_cuda.h"

static void* g_stream = nullptr;

extern "C" {
int gs_init() {
    if (!g_stream) g_stream = allocate_cuda_stream_host(1, 0);
    return g_stream != nullptr;
}
void* gs_allocate(unsigned long long dim) { return allocate_quantum_state_host(dim, 0); }
void gs_initialize(void* s, unsigned long long dim) { initialize_quantum_state_host(s, dim, g_stream, 0); }
void gs_release(void* s) { release_quantum_state_host(s, 0); }
void gs_RX(unsigned t, double a, void* s, unsigned long long dim) { RX_gate_host(t, a, s, dim, g_stream, 0); }
void gs_RY(unsigned t, double a, void* s, unsigned long long dim) { RY_gate_host(t, a, s, dim, g_stream, 0); }
void gs_RZ(unsigned t, double a, void* s, unsigned long long dim) { RZ_gate_host(t, a, s, dim, g_stream, 0); }
void gs_CNOT(unsigned c, unsigned t, void* s, unsigned long long dim) { CNOT_gate_host(c, t, s, dim, g_stream, 0); }
double gs_norm(void* s, unsigned long long dim) { return state_norm_squared_host(s, dim, g_stream, 0); }
}
