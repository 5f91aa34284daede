// Library context, error state and logging.
#include "internal.h"

#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace {

thread_local int g_last_error = BML_B200_OK;
int g_verbose = 1;
int g_requested_device = -1;
unsigned long long g_launches = 0;
cudaEvent_t g_events[64];
bool g_events_ready = false;

B200Context g_ctx;
bool g_ctx_ready = false;
bool g_ctx_failed = false;
std::mutex g_ctx_mutex;

} // namespace

void b200_count_launch() { ++g_launches; }

void b200_set_error(int status, const char *fmt, ...)
{
    g_last_error = status;
    if (!g_verbose)
        return;
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "[bml_b200 error %d: %s] ", status, bml_b200_error_string(status));
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
}

int b200_get_error() { return g_last_error; }

int b200_swap_verbose(int on)
{
    const int old = g_verbose;
    g_verbose = on;
    return old;
}

bool b200_cuda_ok(cudaError_t err, const char *what, const char *file, int line)
{
    if (err == cudaSuccess)
        return true;
    if (g_ctx_failed)
        return false;
    b200_set_error(BML_B200_ERR_CUDA, "%s failed at %s:%d: %s", what, file, line,
                   cudaGetErrorString(err));
    return false;
}

B200Context *b200_ctx()
{
    if (g_ctx_ready)
        return &g_ctx;
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    if (g_ctx_ready)
        return &g_ctx;
    if (g_ctx_failed)
    {
        b200_set_error(BML_B200_ERR_NO_DEVICE, "no usable CUDA device");
        return nullptr;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
    {
        g_ctx_failed = true;
        b200_set_error(BML_B200_ERR_NO_DEVICE, "no usable CUDA device (%s)",
                       e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
        return nullptr;
    }
    memset(&g_ctx, 0, sizeof(g_ctx));
    if (g_requested_device >= 0 && !CUDA_OK(cudaSetDevice(g_requested_device)))
        return nullptr;
    if (!CUDA_OK(cudaGetDevice(&g_ctx.device)))
        return nullptr;
    cudaDeviceProp prop;
    if (!CUDA_OK(cudaGetDeviceProperties(&prop, g_ctx.device)))
        return nullptr;
    if (prop.major < 10)
    {
        g_ctx_failed = true;
        b200_set_error(BML_B200_ERR_NO_DEVICE,
                       "device %d (%s, sm_%d%d) is not an sm_100 part; the kernels are built for sm_100a only",
                       g_ctx.device, prop.name, prop.major, prop.minor);
        return nullptr;
    }
    g_ctx.sm_count = prop.multiProcessorCount;
    g_ctx.smem_optin = prop.sharedMemPerBlockOptin;
    if (!CUDA_OK(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking)))
        return nullptr;
    // Matrices and scratch come from the device's stream-ordered pool on the
    // library stream; the pool keeps freed memory for reuse (no release
    // threshold), so SP2's per-call temporaries of a few GB cost neither a
    // device synchronisation nor a trip to the driver after the first call.
    {
        cudaMemPool_t pool;
        if (!CUDA_OK(cudaDeviceGetDefaultMemPool(&pool, g_ctx.device)))
            return nullptr;
        unsigned long long keep = ~0ull;
        if (!CUDA_OK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)))
            return nullptr;
    }
    if (!CUDA_OK(cudaMallocHost(&g_ctx.pinned, 65536)))
        return nullptr;
    if (!CUDA_OK(cudaMalloc(&g_ctx.d_small, 65536)))
        return nullptr;
    g_ctx_ready = true;
    return &g_ctx;
}

void *b200_scratch(size_t bytes)
{
    B200Context *c = b200_ctx();
    if (!c)
        return nullptr;
    if (bytes <= c->scratch_bytes)
        return c->scratch;
    // Grow geometrically.  The old arena may still be in use by queued
    // kernels: it is freed in stream order, after them.
    if (c->scratch)
        cudaFreeAsync(c->scratch, c->stream);
    c->scratch = nullptr;
    c->scratch_bytes = 0;
    size_t want = bytes + bytes / 4 + (1 << 20);
    if (cudaMallocAsync(&c->scratch, want, c->stream) != cudaSuccess)
    {
        cudaGetLastError();
        b200_set_error(BML_B200_ERR_ALLOC, "device scratch of %zu bytes", want);
        c->scratch = nullptr;
        return nullptr;
    }
    c->scratch_bytes = want;
    return c->scratch;
}

bool b200_sync()
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    return CUDA_OK(cudaStreamSynchronize(c->stream));
}

// ---------------------------------------------------------------------------
// C ABI: status and housekeeping
// ---------------------------------------------------------------------------
extern "C" {

int bml_b200_last_error(void) { return g_last_error; }

void bml_b200_clear_error(void) { g_last_error = BML_B200_OK; }

void bml_b200_set_verbose(int on) { g_verbose = on; }

const char *bml_b200_error_string(int status)
{
    switch (status)
    {
    case BML_B200_OK: return "ok";
    case BML_B200_ERR_NO_DEVICE: return "no usable CUDA device";
    case BML_B200_ERR_CUDA: return "CUDA runtime error";
    case BML_B200_ERR_INVALID: return "invalid argument";
    case BML_B200_ERR_UNSUPPORTED: return "unsupported matrix type or precision";
    case BML_B200_ERR_ROW_OVERFLOW: return "Number of non-zeroes per row > M, Increase M";
    case BML_B200_ERR_ALLOC: return "allocation failed";
    case BML_B200_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
    }
}

int bml_b200_synchronize(void) { return b200_sync() ? BML_B200_OK : b200_get_error(); }

int bml_b200_device_info(int *sm_count, int *device)
{
    B200Context *c = b200_ctx();
    if (!c)
        return b200_get_error();
    if (sm_count)
        *sm_count = c->sm_count;
    if (device)
        *device = c->device;
    return BML_B200_OK;
}

void bml_init(void) { (void) b200_ctx(); }

int bml_getNRanks(void) { return 1; }

int bml_getMyRank(void) { return 0; }

int bml_printRank(void) { return 1; }

int bml_b200_set_device(int device)
{
    if (g_ctx_ready && g_ctx.device != device)
    {
        b200_set_error(BML_B200_ERR_INVALID, "set_device(%d) after the library started on device %d",
                       device, g_ctx.device);
        return BML_B200_ERR_INVALID;
    }
    g_requested_device = device;
    return BML_B200_OK;
}

unsigned long long bml_b200_launch_count(void) { return g_launches; }

int bml_b200_event_record(int slot)
{
    B200Context *c = b200_ctx();
    if (!c)
        return b200_get_error();
    if (slot < 0 || slot >= 64)
        return BML_B200_ERR_INVALID;
    if (!g_events_ready)
    {
        for (int e = 0; e < 64; ++e)
            if (!CUDA_OK(cudaEventCreate(&g_events[e])))
                return b200_get_error();
        g_events_ready = true;
    }
    return CUDA_OK(cudaEventRecord(g_events[slot], c->stream)) ? BML_B200_OK : b200_get_error();
}

int bml_b200_event_elapsed(int a, int b, float *ms)
{
    if (!g_events_ready || a < 0 || b < 0 || a >= 64 || b >= 64 || !ms)
        return BML_B200_ERR_INVALID;
    if (!CUDA_OK(cudaEventSynchronize(g_events[b])) ||
        !CUDA_OK(cudaEventElapsedTime(ms, g_events[a], g_events[b])))
        return b200_get_error();
    return BML_B200_OK;
}

void bml_shutdown(void)
{
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    if (!g_ctx_ready)
        return;
    if (g_ctx.scratch)
        cudaFreeAsync(g_ctx.scratch, g_ctx.stream);
    cudaStreamSynchronize(g_ctx.stream);
    if (g_ctx.d_small)
        cudaFree(g_ctx.d_small);
    if (g_ctx.pinned)
        cudaFreeHost(g_ctx.pinned);
    cudaStreamDestroy(g_ctx.stream);
    memset(&g_ctx, 0, sizeof(g_ctx));
    g_ctx_ready = false;
}

// Logging with the reference's level names; an ERROR is reported and recorded
// but never terminates the process (the reference exits, bml_logger.c:111-115).
static void b200_vlog(bml_log_level_t level, const char *file, int line,
                      const char *format, va_list ap)
{
    if (level == BML_LOG_DEBUG)
        return;
    FILE *out = level >= BML_LOG_WARNING ? stderr : stdout;
    if (level == BML_LOG_ERROR)
        g_last_error = BML_B200_ERR_INVALID;
    if (file)
        fprintf(out, "[%s:%d] ", file, line);
    if (level == BML_LOG_WARNING)
        fprintf(out, "WARNING ");
    if (level == BML_LOG_ERROR)
        fprintf(out, "ERROR ");
    vfprintf(out, format, ap);
    fflush(out);
}

void bml_log(bml_log_level_t log_level, char *format, ...)
{
    va_list ap;
    va_start(ap, format);
    b200_vlog(log_level, nullptr, 0, format, ap);
    va_end(ap);
}

void bml_log_location(bml_log_level_t log_level, char *filename, int linenumber,
                      char *format, ...)
{
    va_list ap;
    va_start(ap, format);
    b200_vlog(log_level, filename, linenumber, format, ap);
    va_end(ap);
}

char *bml_version(void)
{
    static char v[] = "2.4.0-b200";
    return v;
}

void bml_print_version(void)
{
    printf("bml version %s (B200 sm_100a ELLPACK/ELLBLOCK path)\n", bml_version());
}

} // extern "C"
