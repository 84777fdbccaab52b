// A no-allocation form of the one-plane stage (nssb_bm3d_plane_stage_noalloc).
//
// Who needs it: hosts that cannot call cudaMalloc/cudaFree while they run --
// a video pipeline whose device memory is owned by its own frame pool and
// budgeted once at start-up, or a latency-critical loop where an allocation
// would block or synchronise the device. Such a caller passes its input and
// output planes and gets the stage's work done without the library
// allocating anything.
//
// How: every scratch buffer the stage needs (match lists, group sizes and the
// fixed-point num / origin-weight sums) is carved from one file-scope device
// array of kNoAllocBytes, which every GPU that loads this library holds until
// the process exits. The array's name in host code is only a host-side
// stand-in, never a device address: its device address is looked up once per
// device with cudaGetSymbolAddress (with that device current) on the first
// call on that device, and passed to the kernels; the same set-up uploads the
// generic group kernel's DCT tables to the device. Make that first call
// before any stream capture. A set-up that fails (under capture, say) is not
// remembered: the next call on that device tries again.
//
// All calls share the array and it keeps the last call's contents: each call
// clears the sums it accumulates into before use. Calls that overlap on the
// GPU (on different streams, or from different host threads) race on the
// array; serialise them.
#include "engine.hpp"

#include <mutex>
#include <string>

namespace nssb {
namespace {

// Limits of the no-allocation stage: planes up to 2 MiPx (1920x1088 fits),
// up to 256 Ki references and 1 Mi match entries (references x group).
constexpr size_t kNoAllocMaxPixels = size_t(1) << 21;
constexpr size_t kNoAllocMaxJobs = size_t(1) << 18;
constexpr size_t kNoAllocMaxEntries = size_t(1) << 20;
constexpr size_t kNumBytes = kNoAllocMaxPixels * sizeof(long long);
constexpr size_t kWsumBytes = kNoAllocMaxPixels * sizeof(long long);
constexpr size_t kPosBytes = kNoAllocMaxEntries * sizeof(int32_t);
constexpr size_t kCountBytes = kNoAllocMaxJobs * sizeof(int32_t);
constexpr size_t kNoAllocBytes = kNumBytes + kWsumBytes + kPosBytes + kCountBytes;  // 37 MiB
static_assert(kNumBytes % 256 == 0 && kWsumBytes % 256 == 0 && kPosBytes % 256 == 0, "256-byte carving");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices];  // set only once a set-up succeeded

unsigned char* scratch_for_current_device() {
    int dev = 0;
    NSSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw std::invalid_argument("nss_cuda: device index beyond the no-allocation table");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        ensure_group_tables();
        void* p = nullptr;
        NSSB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        if (!p) throw CudaError("nss_cuda: cudaGetSymbolAddress gave no address for the stage scratch");
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_scratch_ptr[dev];
}

}  // namespace

void plane_stage_noalloc(const float* src, const float* ref, float* dst, int64_t stride, int w, int h,
                         const StageParams& sp, cudaStream_t stream) {
    const size_t pixels = (size_t)stride * (size_t)h;
    const size_t jobs = (size_t)grid_count(w, sp.block, sp.step) * (size_t)grid_count(h, sp.block, sp.step);
    const size_t entries = jobs * (size_t)sp.group;
    if (pixels > kNoAllocMaxPixels || jobs > kNoAllocMaxJobs || entries > kNoAllocMaxEntries) {
        throw std::invalid_argument(
            "nss_cuda: nssb_bm3d_plane_stage_noalloc handles at most " + std::to_string(kNoAllocMaxPixels) +
            " plane elements (stride x height), " + std::to_string(kNoAllocMaxJobs) + " references and " +
            std::to_string(kNoAllocMaxEntries) + " match entries; this call needs " + std::to_string(pixels) + ", " +
            std::to_string(jobs) + " and " + std::to_string(entries));
    }
    if (group_filter_scratch_floats(sp.block, sp.group, ref != nullptr) != 0) {
        throw std::invalid_argument("nss_cuda: nssb_bm3d_plane_stage_noalloc does not take block " +
                                    std::to_string(sp.block) + " with group " + std::to_string(sp.group) +
                                    " (the group cube needs global scratch)");
    }
    unsigned char* base = scratch_for_current_device();
    if (sp.sigma == 0.f) {
        NSSB_CUDA(cudaMemcpy2DAsync(dst, stride * 4, src, stride * 4, w * 4, h, cudaMemcpyDeviceToDevice, stream));
        return;
    }
    long long* num = reinterpret_cast<long long*>(base);
    long long* wsum = reinterpret_cast<long long*>(base + kNumBytes);
    int32_t* pos = reinterpret_cast<int32_t*>(base + kNumBytes + kWsumBytes);
    int32_t* count = reinterpret_cast<int32_t*>(base + kNumBytes + kWsumBytes + kPosBytes);
    // the previous call's sums are still there: start from zero
    NSSB_CUDA(cudaMemsetAsync(num, 0, pixels * sizeof(long long), stream));
    NSSB_CUDA(cudaMemsetAsync(wsum, 0, pixels * sizeof(long long), stream));
    launch_match_spatial(ref ? ref : src, stride, w, h, sp.block, sp.step, sp.bm_range, sp.group, pos, nullptr, count,
                         stream);
    GroupIO io{};
    io.src[0] = src;
    io.ref[0] = ref;
    io.stride = stride;
    io.ref_stride = stride;
    io.num[0] = num;
    io.wsum[0] = wsum;
    io.acc_stride = stride;
    launch_group_filter(io, w, h, pos, nullptr, count, (int)jobs, sp.block, sp.group, sp.sigma, ref != nullptr,
                        nullptr, 0, stream);
    launch_finish(num, wsum, stride, src, stride, dst, stride, w, h, sp.block, stream);
}

}  // namespace nssb
