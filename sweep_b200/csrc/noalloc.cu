// noalloc.cu -- sweep_b200_acoustic_forward_noalloc: a 2-D acoustic forward
// (records only) whose scratch lives in this file's static device array, for
// callers that cannot allocate device memory: code that runs where
// cudaMalloc is not allowed or not wanted -- inside another library's memory
// manager, a real-time loop that must not allocate, or a host process whose
// device memory is already fully handed out.
//
// Properties a caller must know:
//   * the array (kNoAllocScratchBytes) exists on every GPU that loads this
//     library, from load to process exit;
//   * every call synchronizes its stream (the source / receiver tables are
//     staged through host memory, the error word is read back), so no call
//     can run under stream capture;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current);
//   * every call on a device uses the same array: calls that overlap on the
//     GPU race and corrupt each other; run them one after the other.  Calls
//     from this process are serialised by one process-wide lock held for the
//     whole call (calls on different GPUs too, since they share the static
//     host staging buffers), so the race concerns work that reaches the
//     array some other way, e.g. another copy of this library loaded into
//     the process;
//   * the address looked up on a device's first call is kept for the life of
//     the process: cudaDeviceReset on that device after the entry point has
//     been used is not supported (the module may load at another address);
//   * each call clears the fields that must start at zero, so a call never
//     sees what the previous one left behind;
//   * no cudaMalloc, cudaFree or any other allocating routine is called; host
//     staging of the source/receiver tables uses fixed static buffers, so the
//     number of events and tiles is bounded too.
#include <mutex>

#include "acoustic2d.cuh"

namespace {

constexpr long long kNoAllocScratchBytes = 64LL << 20;   // 64 MiB per GPU
constexpr int kMaxKeys = 1 << 16;                          // shots x tiles
constexpr int kMaxEvents = 1 << 15;                        // shots x (sources | receivers)
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// One process-wide lock over the static host staging buffers and the
// per-device address table.
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

int32_t h_loc_src[2 * kMaxEvents], h_loc_rec[2 * kMaxEvents];
int32_t h_off_src[kMaxKeys + 1], h_off_rec[kMaxKeys + 1], h_fill[kMaxKeys + 1], h_order[kMaxKeys + 1];
int2 h_ev_src[kMaxEvents], h_ev_rec[kMaxEvents];

int current_device()
{
    int dev = -1;
    SWEEP_CUDA(cudaGetDevice(&dev));
    SWEEP_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal %d out of range", dev);
    return dev;
}

// Device address of device `dev`'s scratch array (`dev` current), looked up
// once per device; the caller holds g_mutex.
void* scratch_of_device(int dev)
{
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        SWEEP_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        SWEEP_REQUIRE(p != nullptr, "cudaGetSymbolAddress returned a null address");
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace

using namespace sweep;

extern "C" SWEEP_B200_API int sweep_b200_acoustic_forward_noalloc(const sweep_acoustic_desc* d, float* record,
                                                                 void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        SWEEP_REQUIRE(d->ndim == 2, "acoustic forward_noalloc: only 2-D (ndim 2) is built (got %d)", d->ndim);
        const int64_t need = a2d::forward_only_bytes(d);
        SWEEP_REQUIRE(need <= kNoAllocScratchBytes,
                      "acoustic forward_noalloc: the problem needs %lld bytes of scratch, more than the "
                      "%lld-byte static array; use sweep_b200_acoustic_forward with a caller workspace",
                      (long long)need, (long long)kNoAllocScratchBytes);
        int64_t nkey, nes, ner;
        a2d::stage_sizes(d, &nkey, &nes, &ner);
        SWEEP_REQUIRE(nkey <= kMaxKeys + 1 && nes <= kMaxEvents && ner <= kMaxEvents,
                      "acoustic forward_noalloc: at most %d shot-tiles and %d sources / receivers "
                      "(got %lld, %lld, %lld)", kMaxKeys, kMaxEvents, (long long)nkey - 1,
                      (long long)nes, (long long)ner);
        std::lock_guard<std::mutex> lock(g_mutex);
        void* ws = scratch_of_device(current_device());
        const a2d::HostStage stage{h_loc_src, h_loc_rec, h_off_src, h_off_rec, h_ev_src, h_ev_rec, h_fill, h_order};
        a2d::forward_with(d, SWEEP_MEM_BOUNDARY, 0, record, nullptr, ws, kNoAllocScratchBytes, static_cast<cudaStream_t>(stream),
                          &stage, nullptr, 0, 0);
    });
}
