// Library-wide plumbing: errors, the stream, launch counting, batch geometry.
#include <atomic>
#include <cstring>
#include <mutex>

#include "cw_internal.cuh"

namespace cw {

static thread_local std::string g_error;
static std::atomic<uint64_t> g_launches{0};
static cudaStream_t g_own_stream = nullptr;
static std::once_flag g_own_once;
static cudaStream_t g_user_stream = nullptr;
static bool g_user_set = false;
// the scope of the entry point running on this thread (Scope)
static thread_local cudaStream_t t_stream = nullptr;
static thread_local bool t_scoped = false;
static thread_local std::string *t_err = nullptr;

static TestFaults g_faults;
const TestFaults &test_faults() { return g_faults; }

void set_error(const std::string &msg) {
    g_error = msg;
    if (t_err) *t_err = msg;
}

int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    return CW_ERR_CUDA;
}

// The library stream: the caller's (cw_set_stream), else one of its own.
static cudaStream_t library_stream() {
    if (g_user_set) return g_user_stream;
    std::call_once(g_own_once, [] { cudaStreamCreateWithFlags(&g_own_stream, cudaStreamNonBlocking); });
    return g_own_stream;
}

cudaStream_t stream() {
    if (t_scoped && t_stream) return t_stream;
    return library_stream();
}

int HandleStream::init(bool adopt) {
    if (adopt && t_scoped && t_stream) {
        stream = t_stream;  // a handle made inside another's call shares its stream
        own = false;
        return CW_OK;
    }
    CW_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own = true;
    return CW_OK;
}

int HandleStream::set(cudaStream_t s) {
    if (s && s == stream) return CW_OK;
    if (stream) CW_CUDA(cudaStreamSynchronize(stream));  // work queued so far finishes first
    if (own && stream) cudaStreamDestroy(stream);
    stream = nullptr;
    own = false;
    if (s) {
        stream = s;
        return CW_OK;
    }
    CW_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own = true;
    return CW_OK;
}

void HandleStream::release() {
    if (own && stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
    stream = nullptr;
    own = false;
}

Scope::Scope(HandleStream *hs) : prev_stream_(t_stream), prev_err_(t_err), prev_set_(t_scoped) {
    t_stream = hs->stream;
    t_err = &hs->err;
    t_scoped = true;
}

Scope::~Scope() {
    t_stream = prev_stream_;
    t_err = prev_err_;
    t_scoped = prev_set_;
}

// The other handle's queued work before this call's, and this call's before
// the other handle's next (one event each way; nothing when they share a stream).
Join::Join(const HandleStream *other) : mine_(stream()), other_(other->stream ? other->stream : library_stream()) {
    if (mine_ == other_) return;
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return;
    cudaEventRecord(e, other_);
    cudaStreamWaitEvent(mine_, e, 0);
    cudaEventDestroy(e);
}

Join::~Join() {
    if (mine_ == other_) return;
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return;
    cudaEventRecord(e, mine_);
    cudaStreamWaitEvent(other_, e, 0);
    cudaEventDestroy(e);
}

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int Geom::init(uint32_t n, const uint32_t *W, const uint32_t *H, const uint32_t *D) {
    if (n == 0) return fail(CW_ERR_CONFIG, "a batch needs at least one history");
    nh = n;
    w.resize(n); h.resize(n); d.resize(n); off.assign(n + 1, 0);
    std::vector<int4> dims(n);
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t a = W[k], b = H[k], c = D ? D[k] : 1;
        if (a == 0 || b == 0 || c == 0 || a > 65535 || b > 65535 || c > 65535)
            return fail(CW_ERR_CONFIG, "invalid grid dimensions (" + std::to_string(a) + "x" + std::to_string(b) +
                                           "x" + std::to_string(c) + ") of history " + std::to_string(k));
        if ((uint64_t)a * b * c >= (1ull << 31))
            return fail(CW_ERR_CONFIG, "history " + std::to_string(k) + " has 2^31 pixels or more");
        w[k] = (int32_t)a; h[k] = (int32_t)b; d[k] = (int32_t)c;
        off[k + 1] = off[k] + (int64_t)a * b * c;
        dims[k] = make_int4((int)a, (int)b, (int)c, 0);
    }
    total = off[n];
    int rc;
    if ((rc = dalloc(&d_dims, n)) != CW_OK) return rc;
    if ((rc = dalloc(&d_off, n + 1)) != CW_OK) return rc;
    CW_CUDA(cudaMemcpy(d_dims, dims.data(), sizeof(int4) * n, cudaMemcpyHostToDevice));
    CW_CUDA(cudaMemcpy(d_off, off.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
    return CW_OK;
}

void Geom::release() {
    dfree(d_dims);
    dfree(d_off);
}

int Plan::build(const std::vector<int64_t> &per, int threads) {
    nh = (uint32_t)per.size();
    items = per;
    blk.assign(nh + 1, 0);
    for (uint32_t k = 0; k < nh; ++k) blk[k + 1] = blk[k] + (int32_t)((per[k] + threads - 1) / threads);
    nblocks = blk[nh];
    // on the device: the prefix, then each block's history (one load for a
    // kernel to find its history)
    table = blk;
    table.resize((size_t)nh + 1 + (size_t)nblocks);
    for (uint32_t k = 0; k < nh; ++k)
        for (int32_t b = blk[k]; b < blk[k + 1]; ++b) table[nh + 1 + (size_t)b] = (int32_t)k;
    if (!d_blk || cap < table.size()) {
        dfree(d_blk);
        int rc = dalloc(&d_blk, table.size());
        if (rc != CW_OK) return rc;
        cap = table.size();
    }
    CW_CUDA(cudaMemcpyAsync(d_blk, table.data(), sizeof(int32_t) * table.size(), cudaMemcpyHostToDevice, stream()));
    return CW_OK;
}

void Plan::release() {
    dfree(d_blk);
    cap = 0;
}

}  // namespace cw

extern "C" {

const char *cw_last_error(void) { return cw::g_error.c_str(); }

int cw_version(void) { return 1; }

int cw_set_stream(void *s) {
    cw::g_user_stream = (cudaStream_t)s;
    cw::g_user_set = s != nullptr;
    return CW_OK;
}

void *cw_get_stream(void) { return (void *)cw::stream(); }

int cw_synchronize(void) {
    // every handle's stream and the library's
    CW_CUDA(cudaDeviceSynchronize());
    return CW_OK;
}

uint64_t cw_launch_count(void) { return cw::g_launches.load(); }

int cw_test_faults(uint64_t wait_ns, int32_t withhold_block, int32_t max_rounds, int32_t skip_tma) {
    if (wait_ns != 0 && (wait_ns < 1000000ull || wait_ns > 2000000000ull))
        return cw::fail(CW_ERR_CONFIG, "a test's wait limit lies between 1 ms and 2 s (0: the default)");
    if (max_rounds < 0) return cw::fail(CW_ERR_CONFIG, "a round limit is not below zero (0: the default)");
    cw::g_faults.wait_ns = wait_ns;
    cw::g_faults.withhold_block = withhold_block < 0 ? -1 : withhold_block;
    cw::g_faults.max_rounds = max_rounds;
    cw::g_faults.skip_tma = skip_tma ? 1 : 0;
    return CW_OK;
}

}  // extern "C"

// Timing on the library stream: events in numbered slots.
namespace {
cudaEvent_t g_events[16] = {};
}

extern "C" int cw_event_record(int32_t slot) {
    if (slot < 0 || slot >= 16) return cw::fail(CW_ERR_CONFIG, "event slots are 0 to 15");
    if (!g_events[slot]) CW_CUDA(cudaEventCreate(&g_events[slot]));
    CW_CUDA(cudaEventRecord(g_events[slot], cw::stream()));
    return CW_OK;
}

extern "C" int cw_event_record_on(void *stream, int32_t slot) {
    if (slot < 0 || slot >= 16) return cw::fail(CW_ERR_CONFIG, "event slots are 0 to 15");
    if (!g_events[slot]) CW_CUDA(cudaEventCreate(&g_events[slot]));
    CW_CUDA(cudaEventRecord(g_events[slot], stream ? (cudaStream_t)stream : cw::stream()));
    return CW_OK;
}

extern "C" int cw_event_elapsed(int32_t a, int32_t b, float *ms) {
    if (a < 0 || a >= 16 || b < 0 || b >= 16 || !g_events[a] || !g_events[b])
        return cw::fail(CW_ERR_CONFIG, "both events must have been recorded");
    CW_CUDA(cudaEventSynchronize(g_events[b]));
    CW_CUDA(cudaEventElapsedTime(ms, g_events[a], g_events[b]));
    return CW_OK;
}

extern "C" int cw_set_device(int32_t device) {
    CW_CUDA(cudaSetDevice(device));
    return CW_OK;
}

#include <cuda_profiler_api.h>

// Bracket a region for a profiler started with profiling off.
extern "C" int cw_profiler_start(void) {
    CW_CUDA(cudaProfilerStart());
    return CW_OK;
}

extern "C" int cw_profiler_stop(void) {
    CW_CUDA(cudaStreamSynchronize(cw::stream()));
    CW_CUDA(cudaProfilerStop());
    return CW_OK;
}
