// capi.cu — version, status strings and the thread-local last-error message
// of libnsph.so.
#include <string>

#include "nsph_internal.cuh"

namespace nsph {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

int fail(int status, const std::string& msg)
{
    set_error(msg);
    return status;
}

int cuda_fail(cudaError_t err, const char* what)
{
    set_error(std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")");
    return NSPH_ERR_CUDA;
}

}  // namespace nsph

extern "C" int nsph_version(void) { return 1; }

extern "C" const char* nsph_status_string(int status)
{
    switch (status) {
        case NSPH_OK: return "ok";
        case NSPH_ERR_INVALID_ARG: return "invalid argument";
        case NSPH_ERR_CAPACITY: return "capacity exceeded";
        case NSPH_ERR_CUDA: return "CUDA error";
        case NSPH_ERR_NOT_BUILT: return "grid not built";
        case NSPH_ERR_OUT_OF_MEMORY: return "out of memory";
        default: return "unknown status";
    }
}

extern "C" const char* nsph_last_error(void) { return nsph::g_last_error.c_str(); }

extern "C" int nsph_build_flags(void)
{
#ifdef NSPH_BOUNDS_CHECK
    return NSPH_BUILD_BOUNDS_CHECK;
#else
    return 0;
#endif
}

extern "C" int nsph_debug_bounds_violations(unsigned long long* count)
{
    nsph::clear_error();
    if (!count) return nsph::fail(NSPH_ERR_INVALID_ARG, "null count");
    unsigned long long total = 0;
    for (unsigned long long v : {nsph::nsph_bounds_read_hashgrid(), nsph::nsph_bounds_read_sph(),
                                 nsph::nsph_bounds_read_contact(), nsph::nsph_bounds_read_shapes(),
                                 nsph::nsph_bounds_read_raycast()}) {
        if (v == ~0ull) return nsph::fail(NSPH_ERR_CUDA, "cannot read the bounds-check counters");
        total += v;
    }
    *count = total;
    return NSPH_OK;
}
