// Internal interfaces of the B200 search backend, shared by the CUDA kernel
// files and the host engine. Everything here is C++; the public surface is the
// C ABI in include/ft_b200.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace ftb {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what);
#define FTB_CHECK(call) ::ftb::cuda_check((call), #call)

// Device pixel layout of a frame stack: n frames of h rows, row pitch `pitch`
// floats (a multiple of 32, so every row starts on a 128-byte boundary, as TMA
// tensor maps require); columns [w, pitch) are never read as image data.
inline int frame_pitch(int w) { return (w + 31) / 32 * 32; }

// ------------------------------------------------------------------ stacking
// A pass plan: the motions are cut into groups whose shifted frame windows fit
// together in shared memory for one output tile (see stack.cu).
struct StackGroup {
    int slot0 = 0;           // first slot of the group in the slot arrays
    int nslots = 0;          // slots (a multiple of the motion block; pads are -1)
    int gdxmin = 0, gdxmax = 0, gdymin = 0, gdymax = 0;  // shift extremes over the group
    int rows_total = 0;      // window rows in shared memory (sum over frames)
    int win0 = 0;            // first per-frame window descriptor of the group
    int rows_fast = 0;       // 1: every block shares its column in every frame (row descriptors)
    int tab_bytes = 0;       // bytes of the group's offset table (a multiple of 16)
};

// Motions are planned in blocks of kMotionBlock slots (one register block of
// the kernel). A block whose motions, in every frame, share the column shift and
// lie within kRowSpread rows of one another is described per frame by one
// 32-bit word: bits 0-15 the window offset of its lowest row, bits 16-23 each
// slot's row above it (2 bits a slot), bits 24-25 the largest of those, and,
// when that is at most 1, bits 26-29 the slots' offsets as a 4-bit pattern;
// bits 30-31 are zero, so a word below 2^24 has every slot on the lowest row.
constexpr int kMotionBlock = 4;
constexpr int kRowSpread = 3;
// The largest row offset a tile shape's kernel takes in a row-descriptor block:
// 1 for the shapes with fewer registers a thread (the 12-row tile and the shared
// maximum), kRowSpread otherwise. The planner cuts blocks to it.
__host__ __device__ constexpr int shape_row_spread(int p, int merge) { return (p == 12 || merge) ? 1 : kRowSpread; }

struct StackWin {            // one frame's window for a group
    int dx0 = 0;             // window x origin relative to the tile (a multiple of 4)
    int dy0 = 0;             // window y origin relative to the tile
    int row0 = 0;            // first shared-memory row of the window
    int rows = 0;            // rows (a multiple of the TMA box height)
};

struct StackConfig {         // one compiled kernel variant
    int ty = 12;             // warps per CTA; they share the tile and split the motions
    int p = 16;              // output rows per tile (and per thread)
    int tile_w = 32;         // output columns per tile (one warp)
    int tile_h() const { return p; }
    int threads() const { return 32 * ty; }
    int wp = 40;             // window pitch in floats
    int bh = 4;              // TMA box height (rows)
    int mblock = 4;          // motions accumulated together in registers
    int merge = 0;           // 0: best/argmax per thread; 1: one shared maximum per tile (atomicMax)
    int rows = 0;            // > 0: the kernel reads row descriptors (blocks sharing a column) whose
                             // row offsets are at most this
    int smem_bytes = 200 * 1024;
};

struct StackPlan {
    int w = 0, h = 0, n = 0, m = 0, min_count = 1, pitch = 0;
    StackConfig cfg;
    std::vector<StackGroup> groups;
    std::vector<StackWin> wins;               // groups x frames
    std::vector<int> slot_motion;             // motion index per slot, -1 = pad
    std::vector<uint16_t> slot_off;           // per group: [frame][slot] shared-memory offsets, or for a
                                              // rows_fast group [frame][block] 32-bit row descriptors
    std::vector<int> slot_off_base;           // per group: start in slot_off (elements)
    std::vector<short2> slot_shift;           // [slot][frame] clamped (dx, dy), for coverage counts
    std::vector<float> inv_sqrt;              // float(1 / sqrt(c)), c = 0..n
    int max_rows = 0;                         // largest rows_total over the groups
    long long max_group_bytes = 0;            // largest windows + offset table of one group
    int max_slots = 0;
    double adds = 0;                          // m * n * w * h
};

// Motion blocks for the planner, flattened: kMotionBlock slots a block, -1 for a
// pad. Motions whose column shifts agree in every frame form a class; a class is
// cut, in index order, into blocks whose rows stay within kRowSpread of one
// another in every frame; blocks whose shifts are close come together (patches
// of about sx x sy pixels at the frame of widest spread).
std::vector<int> motion_order(const int* dx, const int* dy, int m, int n, double sx_px, double sy_px);

// Build a plan for a pass; dx/dy are motion-major (j * n + i) host tables.
StackPlan make_stack_plan(int w, int h, int n, const int* dx, const int* dy, int m, int min_count,
                          const std::vector<int>& order, const StackConfig& cfg);

StackConfig choose_stack_config(int w, int h, int n, int device_smem_optin);

// The maps of a pass whose min_count exceeds its frame count, where no S/N is
// defined: max_snr +0.0f and best_v -1 for `pixels` dense pixels.
void fill_undefined_maps(float* d_max_snr, int* d_best_v, size_t pixels, cudaStream_t s);

// The stacking kernel walked on the CPU over its plan (stack_emulate.cpp);
// frames: n x h x w host floats; outputs h x w.
void emulate_stack_pass(const StackPlan& plan, const float* frames, float* max_snr, int* best_v);

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`, never lowering it: the attribute is process-wide, so setting it
// per launch from several threads (the server's workers) could lower it under
// another thread's launch.
void allow_dynamic_smem(const void* func, size_t bytes);

// Compiled stack kernel shapes: 1 = 32 x 16 tiles (12 warps), 2 = 64 x 8 tiles with
// paired columns (12 warps), 3 = 32 x 8 (16 warps), 4 = 32 x 4 (16 warps),
// 5 = 32 x 16 with one shared maximum per tile (16 warps), 6 = the same with 14 warps,
// 7 = 32 x 12 (16 warps), 8 = 32 x 20 with the shared maximum (16 warps).
constexpr int kStackShapes = 8;
StackConfig stack_shape_config(int shape, int device_smem_optin);
bool stack_shape_fits(const StackConfig& c, int n);
// A process-wide choice for choose_stack_config: 0 = by frame count, else a shape
// (used when its windows fit).
void set_stack_shape(int shape);
int stack_shape();
// Test of the bounded staging wait: every stacking launch's barrier expects
// extra_bytes (> 0) that no copy brings, and its waits give up after
// wait_cycles clock cycles with the error flag set; 0 restores the normal
// launches (no extra bytes, a two-second limit).
void set_wait_test(int extra_bytes, long long wait_cycles);

// Device copy of a plan.
struct StackPlanDev {
    StackGroup* groups = nullptr;
    StackWin* wins = nullptr;
    int* slot_motion = nullptr;
    uint16_t* slot_off = nullptr;
    int* slot_off_base = nullptr;
    short2* slot_shift = nullptr;
    float* inv_sqrt = nullptr;
    int ngroups = 0;
    void upload(const StackPlan& p, cudaStream_t s);
    void release();
    cudaStream_t stream_ = nullptr;
};

// One planned pass of a batch over device frames (n x h x pitch), writing
// max_snr / best_v (h x w, dense). best/arg carry the running maxima between
// launches when a pass is split into group ranges [g0, g1).
struct BatchPass {
    const StackPlan* plan = nullptr;
    const StackPlanDev* dev = nullptr;
    const float* frames = nullptr;
    int g0 = 0, g1 = 0;
    bool first = true, last = true;
    float* best = nullptr;
    int* arg = nullptr;
    float* max_snr = nullptr;
    int* best_v = nullptr;
    int tile_rows0 = 0, tile_rows = 0;  // a band of tile rows only (0 rows: the whole pass)
};

// Device bytes of the descriptors of a batch (a work-queue counter, one tensor
// map and one argument block per pass).
size_t batch_desc_bytes(int npasses);

// All passes of a batch in one persistent launch (one CTA per SM taking
// (pass, tile) items from a queue). The passes must share a kernel shape
// (cfg.ty, cfg.p). d_desc: device buffer of at least batch_desc_bytes bytes.
void stack_launch_batch(const std::vector<BatchPass>& batch, unsigned char* d_desc, size_t desc_bytes, int* d_err,
                        int sms, cudaStream_t s);

}  // namespace ftb
