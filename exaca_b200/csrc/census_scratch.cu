// Census of IntermediateOutputAndCheck (src/CAupdate.cpp:738-808) over cell fields the caller
// already holds in device memory, for callers that must not allocate device memory.
//
// Who cannot allocate: a monitor sampling the progress of solves that are still running (a
// cudaMalloc or cudaFree may synchronise the whole device and stall every solve on it), and a
// serving process whose HBM budget is handed out in full to admitted domains. The pool's own
// census (exaca_pool_census) keeps its accumulator in a buffer it allocated at pool creation and
// reads a pool slot; this variant reads any caller arrays and keeps its working data in the
// fixed file-scope array below instead.
//
// Scratch: kScratchBytes = 26 KiB, for at most kMaxDomains = 256 domains per call. The first
// 256 * 56 bytes hold the copied domain descriptors, the next 256 * 48 bytes one accumulator of six
// 64-bit counters per domain. Every call on a device shares this array and it keeps what the last
// call left in it: each call copies its descriptors in and clears its accumulators to zero before
// the kernel runs. Two calls whose work overlapped on the device would race on the array, so a
// call holds a per-device lock until its stream has drained.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/exaca_b200.h"
#include "exaca_host.hpp"

namespace exaca {

namespace {

constexpr int kMaxDomains = EXACA_CENSUS_MAX_DOMAINS;
constexpr size_t kDescBytes = sizeof(exaca_cell_fields);
constexpr size_t kAccWords = 6;
constexpr size_t kAccOffset = kMaxDomains * kDescBytes;
constexpr size_t kScratchBytes = kAccOffset + kMaxDomains * kAccWords * sizeof(unsigned long long);
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

static_assert(kDescBytes == 56, "exaca_cell_fields is 56 bytes on LP64");
static_assert(sizeof(exaca_census) == kAccWords * sizeof(unsigned long long), "exaca_census is six counters");
static_assert(kScratchBytes == 26624, "26 KiB scratch");

static __device__ __align__(256) unsigned char g_census_scratch[kScratchBytes];

// One accumulator per domain: superheated, undercooled, active, solid, remaining, and the bitwise
// complement of the minimum CritTimeStep of the layer's liquid cells in the active window (so that
// all six start at zero; zero means "no such cell" = ULLONG_MAX once complemented back). Cells of
// the current layer are classified (src/CAupdate.cpp:741-752), liquid cells of any other layer are
// remaining (:754-757); the minimum is taken over the window only (:792-805).
__global__ void __launch_bounds__(kThreads) k_census_cells(const exaca_cell_fields *cells, unsigned long long *acc) {
    const exaca_cell_fields d = cells[blockIdx.y];
    unsigned long long *out = acc + kAccWords * blockIdx.y;
    unsigned long long a[5] = {0, 0, 0, 0, 0};
    unsigned long long neg_mn = 0;
    const long long w_lo = d.window_start, w_hi = d.window_start + d.active_size;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < d.domain_size; c += stride) {
        const int t = d.cell_type[c];
        const int ly = d.layer_id[c];
        const int cts = d.crit_time_step[c];
        if (ly == d.layer) {
            if (t == kLiquid) {
                if (cts > d.cycle)
                    a[0]++;
                else
                    a[1]++;
                const unsigned long long neg = ~(unsigned long long)(long long)cts;
                if (c >= w_lo && c < w_hi && neg > neg_mn)
                    neg_mn = neg;
            }
            else if (t == kActive)
                a[2]++;
            else if (t == kSolid)
                a[3]++;
        }
        else if (t == kLiquid) {
            a[4]++;
        }
    }
    for (int q = 0; q < 5; q++) {
        unsigned long long v = a[q];
        for (int o = 16; o; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v)
            atomicAdd(out + q, v);
    }
    for (int o = 16; o; o >>= 1) {
        unsigned long long v = __shfl_down_sync(0xffffffffu, neg_mn, o);
        neg_mn = v > neg_mn ? v : neg_mn;
    }
    if ((threadIdx.x & 31) == 0 && neg_mn)
        atomicMax(out + 5, neg_mn);
}

struct DeviceScratch {
    std::mutex lock;
    bool ready = false;
    unsigned char *ptr = nullptr; // device address of g_census_scratch on this device
    int num_sms = 0;
};

DeviceScratch g_devices[kMaxDevices];

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw DeviceError(std::string(what) + ": " + cudaGetErrorString(e));
}

// Once per device, with that device current: the scratch array's device address, the SM count,
// and the kernel's module loaded (so later calls do no lazy loading).
void setup(DeviceScratch &s, int device) {
    if (s.ready)
        return;
    void *p = nullptr;
    check(cudaGetSymbolAddress(&p, g_census_scratch), "cudaGetSymbolAddress(census scratch)");
    if (reinterpret_cast<uintptr_t>(p) % 256 != 0)
        throw DeviceError("census scratch is not 256-byte aligned");
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
    cudaFuncAttributes fa;
    check(cudaFuncGetAttributes(&fa, k_census_cells), "cudaFuncGetAttributes(k_census_cells)");
    s.ptr = static_cast<unsigned char *>(p);
    s.num_sms = sms;
    s.ready = true;
}

struct DeviceRestore {
    int prev = -1;
    ~DeviceRestore() {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};

} // namespace

void census_cells(int device, void *stream, const exaca_cell_fields *domains, int n_domains, exaca_census *out) {
    DeviceScratch &s = g_devices[device];
    std::lock_guard<std::mutex> guard(s.lock);
    DeviceRestore restore;
    check(cudaGetDevice(&restore.prev), "cudaGetDevice");
    check(cudaSetDevice(device), "cudaSetDevice");
    setup(s, device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    long long largest = 1;
    for (int i = 0; i < n_domains; i++)
        largest = domains[i].domain_size > largest ? domains[i].domain_size : largest;
    unsigned char *desc = s.ptr;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(s.ptr + kAccOffset);
    try {
        check(cudaMemcpyAsync(desc, domains, n_domains * kDescBytes, cudaMemcpyHostToDevice, st), "descriptor copy");
        check(cudaMemsetAsync(acc, 0, n_domains * kAccWords * sizeof(unsigned long long), st), "accumulator clear");
        long long bx = (4ll * s.num_sms + n_domains - 1) / n_domains;
        const long long need = (largest + kThreads - 1) / kThreads;
        bx = bx < need ? bx : need;
        bx = bx < 1 ? 1 : bx;
        k_census_cells<<<dim3((unsigned)bx, (unsigned)n_domains), kThreads, 0, st>>>(
            reinterpret_cast<const exaca_cell_fields *>(desc), acc);
        check(cudaGetLastError(), "k_census_cells launch");
        check(cudaMemcpyAsync(out, acc, n_domains * sizeof(exaca_census), cudaMemcpyDeviceToHost, st), "census copy");
        check(cudaStreamSynchronize(st), "census stream");
    }
    catch (...) {
        // work of this call may still be queued on the stream: the lock (which keeps other calls off
        // the shared array) is released only once it has drained
        cudaStreamSynchronize(st);
        throw;
    }
    for (int i = 0; i < n_domains; i++)
        out[i].next_cts = ~out[i].next_cts;
}

// Number of usable devices (at most kMaxDevices), or -1 when the CUDA runtime reports none.
int census_device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
        return -1;
    return n < kMaxDevices ? n : kMaxDevices;
}

} // namespace exaca
