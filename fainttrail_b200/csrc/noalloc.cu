// An allocation-free stacking pass, for callers that cannot allocate device
// memory: host applications that hand every byte of HBM to their own arena or
// memory pool and forbid a library from growing it, and latency-bound loops
// that must not block on the allocator. The caller owns the frames and the two
// output maps; the pass's only scratch -- its plan tables (motion groups,
// per-frame windows, shared-memory offsets, shifts, 1/sqrt(c)) and the launch
// descriptors -- lives in a file-scope device array of fixed size that every GPU
// loading this library holds until the process exits. The call copies the
// tables from host memory, launches the pass on the caller's stream,
// synchronises that stream and returns when the pass is complete.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ft_b200.h"
#include "ft_internal.h"

namespace ftb {

void set_thread_error(const std::string& msg);  // capi.cpp: what ft_b200_last_error(NULL) reports

namespace {

// 32 MiB: the plan tables of about 5 million (motion, frame) pairs, e.g. the
// 19,328 motions x 40 frames of a 4096^2 full-frame search need 4.7 MiB.
constexpr size_t kScratchBytes = size_t{32} << 20;
static __device__ __align__(256) unsigned char g_plan_scratch[kScratchBytes];
static __device__ __align__(256) int g_wait_error;

struct DeviceScratch {
    bool ready = false;
    unsigned char* tables = nullptr;  // device address of g_plan_scratch on this device
    int* err = nullptr;               // device address of g_wait_error
    int smem_optin = 0;
    int sms = 0;
};

std::mutex g_mu;
DeviceScratch g_devices[64];

// Once per device, with that device current: the device addresses of the arrays
// (the names are host-side stand-ins in host code and cannot be passed to a kernel).
// The stream must belong to the current device, or the copies and the kernel
// would use another device's arrays.
DeviceScratch& device_scratch(cudaStream_t s) {
    int dev = 0;
    FTB_CHECK(cudaGetDevice(&dev));
    if (s) {
        int sdev = -1;
        FTB_CHECK(cudaStreamGetDevice(s, &sdev));
        if (sdev != dev)
            throw std::runtime_error("stack pass: the stream belongs to device " + std::to_string(sdev) +
                                     ", not to the current device " + std::to_string(dev));
    }
    if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceScratch& d = g_devices[dev];
    if (!d.ready) {
        FTB_CHECK(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.tables), g_plan_scratch));
        FTB_CHECK(cudaGetSymbolAddress(reinterpret_cast<void**>(&d.err), g_wait_error));
        FTB_CHECK(cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        FTB_CHECK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
        d.ready = true;
    }
    return d;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

}  // namespace ftb

extern "C" int ft_b200_stack_dev_noalloc(const float* d_frames, int width, int height, int pitch, int nframes,
                                         const int* dx, const int* dy, int motions, int min_count, float* d_max_snr,
                                         int* d_best_v, void* cuda_stream) {
    using namespace ftb;
    try {
        if (!d_frames || !dx || !dy || !d_max_snr || !d_best_v) throw std::runtime_error("stack pass: missing arguments");
        if (nframes < 1 || width < 1 || height < 1 || motions < 1) throw std::runtime_error("stack pass: empty pass");
        if (min_count < 1) throw std::runtime_error("stack pass: min_count must be at least 1");
        if (pitch < width || (pitch * 4) % 16 != 0 || reinterpret_cast<uintptr_t>(d_frames) % 16 != 0)
            throw std::runtime_error("stack pass: device frames need a 16-byte aligned base and row pitch");
        cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
        DeviceScratch& d = device_scratch(s);
        if (min_count > nframes) {  // no S/N is defined anywhere
            fill_undefined_maps(d_max_snr, d_best_v, static_cast<size_t>(width) * height, s);
            FTB_CHECK(cudaStreamSynchronize(s));
            return FT_B200_OK;
        }
        const StackConfig cfg = choose_stack_config(width, height, nframes, d.smem_optin);
        StackPlan plan = make_stack_plan(width, height, nframes, dx, dy, motions, min_count,
                                         motion_order(dx, dy, motions, nframes, 4.0, 4.0), cfg);
        plan.pitch = pitch;
        // the plan tables, one after another at 256-byte boundaries in the array
        struct Part {
            const void* src;
            size_t bytes;
            size_t off;
        };
        std::vector<Part> parts = {
            {plan.groups.data(), plan.groups.size() * sizeof(StackGroup), 0},
            {plan.wins.data(), plan.wins.size() * sizeof(StackWin), 0},
            {plan.slot_motion.data(), plan.slot_motion.size() * sizeof(int), 0},
            {plan.slot_off.data(), plan.slot_off.size() * sizeof(uint16_t), 0},
            {plan.slot_off_base.data(), plan.slot_off_base.size() * sizeof(int), 0},
            {plan.slot_shift.data(), plan.slot_shift.size() * sizeof(short2), 0},
            {plan.inv_sqrt.data(), plan.inv_sqrt.size() * sizeof(float), 0}};
        size_t used = 0;
        for (Part& p : parts) {
            p.off = used;
            used += align256(p.bytes);
        }
        const size_t desc_off = used;  // the launch descriptors follow the tables
        used += align256(batch_desc_bytes(1));
        if (used > kScratchBytes)
            throw std::runtime_error("stack pass: its plan tables need " + std::to_string((used + 1048575) >> 20) +
                                     " MiB; the allocation-free entry point holds at most " +
                                     std::to_string(kScratchBytes >> 20) +
                                     " MiB (fewer motions x frames per call, or ft_b200_stack_dev)");
        for (const Part& p : parts)
            if (p.bytes) FTB_CHECK(cudaMemcpyAsync(d.tables + p.off, p.src, p.bytes, cudaMemcpyHostToDevice, s));
        FTB_CHECK(cudaMemsetAsync(d.err, 0, sizeof(int), s));  // the wait-error flag starts at zero every call
        StackPlanDev view;  // points into the array; never released
        view.groups = reinterpret_cast<StackGroup*>(d.tables + parts[0].off);
        view.wins = reinterpret_cast<StackWin*>(d.tables + parts[1].off);
        view.slot_motion = reinterpret_cast<int*>(d.tables + parts[2].off);
        view.slot_off = reinterpret_cast<uint16_t*>(d.tables + parts[3].off);
        view.slot_off_base = reinterpret_cast<int*>(d.tables + parts[4].off);
        view.slot_shift = reinterpret_cast<short2*>(d.tables + parts[5].off);
        view.inv_sqrt = reinterpret_cast<float*>(d.tables + parts[6].off);
        view.ngroups = static_cast<int>(plan.groups.size());
        BatchPass bp;
        bp.plan = &plan;
        bp.dev = &view;
        bp.frames = d_frames;
        bp.g0 = 0;
        bp.g1 = view.ngroups;
        bp.max_snr = d_max_snr;
        bp.best_v = d_best_v;
        stack_launch_batch({bp}, d.tables + desc_off, kScratchBytes - desc_off, d.err, d.sms, s);
        int err = 0;
        FTB_CHECK(cudaMemcpyAsync(&err, d.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        FTB_CHECK(cudaStreamSynchronize(s));
        if (err) throw std::runtime_error("stack pass: a device wait timed out");
        return FT_B200_OK;
    } catch (const std::exception& e) {
        set_thread_error(e.what());
        return FT_B200_ERROR;
    }
}
