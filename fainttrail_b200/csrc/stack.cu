// Shift-and-stack with per-pixel max-S/N and argmax, for sm_100a.
//
// Contract (FaintTrail backend.hpp:10-40, CPU reference backend_cpu.cpp:77-204):
// for output pixel p and motion j, S_j(p) = (sum over covering frames i, in
// ascending i, of g_i(p + d_ji)) * float(1/sqrt(c)); undefined if c < min_count;
// max_snr = max_j S_j with ties to the lowest j, best_v = argmax or -1; non-finite
// maxima become 0. Results are bit-identical to the CPU backend: every sum starts
// at +0.0f and adds the frames in ascending order with round-to-nearest adds and
// no fused multiply-add.
//
// Design (B200):
//  * One CTA owns a 32 x TH output tile. The motions are cut (host planner) into
//    groups whose shifted windows of all n frames fit in shared memory at once;
//    the CTA walks every group for its tile, so the frames are read from HBM/L2
//    once per group and every staged float feeds (motions in the group) adds.
//  * Windows are staged by TMA (cp.async.bulk.tensor, no multicast) with zero
//    fill outside the frame. A zero from outside the frame adds +0.0f, which is
//    bit-identical to skipping the frame: the running sum starts at +0.0f and a
//    round-to-nearest sum of anything but two -0.0f is never -0.0f. The coverage
//    count c is therefore the only per-frame bookkeeping, and tiles whose group
//    shifts stay inside the frame (almost all) use c = n without counting.
//  * Each thread owns P rows of one column (lanes run along x, so every shared
//    load of a warp is 32 consecutive words: no bank conflicts) and M motions in
//    registers; the per-(motion, frame) window offset comes from a 16-bit table
//    staged with the windows.
//  * The running maximum uses the order-independent rule (larger S/N, or equal
//    S/N and lower motion index), which equals the reference's ascending strict
//    scan whatever order the groups are visited in.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <math_constants.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <unordered_map>

#include "ft_internal.h"

namespace ftb {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string("CUDA: ") + what + ": " + cudaGetErrorString(e));
}

void fill_undefined_maps(float* d_max_snr, int* d_best_v, size_t pixels, cudaStream_t s) {
    FTB_CHECK(cudaMemsetAsync(d_max_snr, 0, sizeof(float) * pixels, s));     // +0.0f
    FTB_CHECK(cudaMemsetAsync(d_best_v, 0xff, sizeof(int) * pixels, s));     // -1
}

void allow_dynamic_smem(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    FTB_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = limit[{dev, func}];
    if (bytes <= cur) return;
    FTB_CHECK(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    cur = bytes;
}

// ------------------------------------------------------------------ host plan

std::vector<int> motion_order(const int* dx, const int* dy, int m, int n, double sx_px, double sy_px) {
    constexpr int M = kMotionBlock;
    std::vector<int> out;
    if (m <= 0 || n <= 0) return out;
    auto DX = [&](int j, int i) { return dx[static_cast<size_t>(j) * n + i]; };
    auto DY = [&](int j, int i) { return dy[static_cast<size_t>(j) * n + i]; };
    // the frame whose shifts spread most (for straight tracks: the frame furthest
    // from the reference epoch) decides the order of the blocks
    int ie = 0;
    long long best = -1;
    for (int i = 0; i < n; ++i) {
        int lo = INT32_MAX, hi = INT32_MIN;
        for (int j = 0; j < m; ++j) {
            lo = std::min({lo, DX(j, i), DY(j, i)});
            hi = std::max({hi, DX(j, i), DY(j, i)});
        }
        if (static_cast<long long>(hi) - lo > best) {
            best = static_cast<long long>(hi) - lo;
            ie = i;
        }
    }
    // classes of motions whose column shifts agree in every frame (for the
    // velocity lattice: equal vx), by a hash of the dx row, checked row by row
    std::vector<int> cls(static_cast<size_t>(m)), rep, chain;
    std::unordered_map<uint64_t, int> by_hash;
    for (int j = 0; j < m; ++j) {
        uint64_t hsh = 1469598103934665603ull;
        for (int i = 0; i < n; ++i) {
            hsh ^= static_cast<uint32_t>(DX(j, i));
            hsh *= 1099511628211ull;
        }
        auto it = by_hash.find(hsh);
        int c = -1;
        if (it != by_hash.end())
            for (int k = it->second; k >= 0 && c < 0; k = chain[static_cast<size_t>(k)])
                if (std::memcmp(dx + static_cast<size_t>(rep[static_cast<size_t>(k)]) * n, dx + static_cast<size_t>(j) * n,
                                sizeof(int) * static_cast<size_t>(n)) == 0)
                    c = k;
        if (c < 0) {
            c = static_cast<int>(rep.size());
            rep.push_back(j);
            chain.push_back(it != by_hash.end() ? it->second : -1);
            by_hash[hsh] = c;
        }
        cls[static_cast<size_t>(j)] = c;
    }
    std::vector<std::vector<int>> members(rep.size());
    for (int j = 0; j < m; ++j) members[static_cast<size_t>(cls[static_cast<size_t>(j)])].push_back(j);
    // each class in index order (for the lattice: ascending vy), cut into blocks
    // whose rows stay within kRowSpread of one another in every frame
    std::vector<std::array<int, M>> blocks;
    std::vector<int> lo(static_cast<size_t>(n)), hi(static_cast<size_t>(n));
    for (const std::vector<int>& mem : members) {
        std::array<int, M> cur;
        int cnt = 0;
        auto close = [&]() {
            for (int k = cnt; k < M; ++k) cur[static_cast<size_t>(k)] = -1;
            blocks.push_back(cur);
            cnt = 0;
        };
        for (int j : mem) {
            bool fits = cnt > 0 && cnt < M;
            for (int i = 0; i < n && fits; ++i) {
                const int v = DY(j, i);
                fits = std::max(hi[static_cast<size_t>(i)], v) - std::min(lo[static_cast<size_t>(i)], v) <= kRowSpread;
            }
            if (!fits && cnt > 0) close();
            if (cnt == 0)
                for (int i = 0; i < n; ++i) lo[static_cast<size_t>(i)] = hi[static_cast<size_t>(i)] = DY(j, i);
            for (int i = 0; i < n; ++i) {
                lo[static_cast<size_t>(i)] = std::min(lo[static_cast<size_t>(i)], DY(j, i));
                hi[static_cast<size_t>(i)] = std::max(hi[static_cast<size_t>(i)], DY(j, i));
            }
            cur[static_cast<size_t>(cnt++)] = j;
        }
        if (cnt > 0) close();
    }
    // tables without that structure (few motions share a column, so most blocks
    // would be padding) are packed densely instead: consecutive motions of the
    // patch order below form the blocks, whose frames then read four offsets each
    const size_t slots = blocks.size() * M;
    if (slots - static_cast<size_t>(m) > static_cast<size_t>(m) / 10) {
        std::vector<int> ord(static_cast<size_t>(m));
        std::iota(ord.begin(), ord.end(), 0);
        auto kxm = [&](int j) { return static_cast<long long>(std::floor(DX(j, ie) / sx_px)); };
        auto kym = [&](int j) { return static_cast<long long>(std::floor(DY(j, ie) / sy_px)); };
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
            if (kxm(a) != kxm(b)) return kxm(a) < kxm(b);
            if (kym(a) != kym(b)) return kym(a) < kym(b);
            if (DY(a, ie) != DY(b, ie)) return DY(a, ie) < DY(b, ie);
            return DX(a, ie) < DX(b, ie);
        });
        blocks.clear();
        for (size_t q = 0; q < ord.size(); q += M) {
            std::array<int, M> b;
            for (int k = 0; k < M; ++k) b[static_cast<size_t>(k)] = q + k < ord.size() ? ord[q + k] : -1;
            blocks.push_back(b);
        }
    }
    // blocks whose shifts are close come together: patches of about sx x sy
    // pixels at frame ie, visited column by column (a group then grows in dy,
    // limited only by shared memory, while its dx spread stays within the window
    // pitch), row-major inside a patch
    auto ex = [&](const std::array<int, M>& b) { return DX(b[0], ie); };
    auto ey = [&](const std::array<int, M>& b) { return DY(b[0], ie); };
    auto kx = [&](const std::array<int, M>& b) { return static_cast<long long>(std::floor(ex(b) / sx_px)); };
    auto ky = [&](const std::array<int, M>& b) { return static_cast<long long>(std::floor(ey(b) / sy_px)); };
    std::stable_sort(blocks.begin(), blocks.end(), [&](const std::array<int, M>& a, const std::array<int, M>& b) {
        if (kx(a) != kx(b)) return kx(a) < kx(b);
        if (ky(a) != ky(b)) return ky(a) < ky(b);
        if (ey(a) != ey(b)) return ey(a) < ey(b);
        return ex(a) < ex(b);
    });
    out.reserve(blocks.size() * M);
    for (const auto& b : blocks) out.insert(out.end(), b.begin(), b.end());
    return out;
}

namespace {
inline int floor4(int v) { return (v >> 2) * 4; }  // arithmetic shift: floor for negatives too
inline int roundup(int v, int q) { return (v + q - 1) / q * q; }
}  // namespace

namespace {
std::atomic<int> g_shape{0};
// a test of the bounded staging wait: extra bytes no copy brings, and the wait's limit
std::atomic<int> g_wait_extra{0};
std::atomic<long long> g_wait_cycles{4000000000LL};
}

void set_wait_test(int extra_bytes, long long wait_cycles) {
    if (extra_bytes < 0 || extra_bytes > (1 << 20) || (extra_bytes > 0 && wait_cycles < 1000))
        throw std::runtime_error("wait test: extra bytes in [0, 1 MiB] and a limit of at least 1000 cycles");
    g_wait_cycles = extra_bytes > 0 ? wait_cycles : 4000000000LL;
    g_wait_extra = extra_bytes;
}

void set_stack_shape(int shape) {
    if (shape < 0 || shape > kStackShapes) throw std::runtime_error("stack: unknown tile shape");
    g_shape = shape;
}

int stack_shape() { return g_shape; }

StackConfig stack_shape_config(int shape, int smem_optin) {
    StackConfig c;
    c.mblock = 4;  // motions per register block
    c.bh = 4;
    c.smem_bytes = std::min(smem_optin - 1024, 224 * 1024);
    switch (shape) {
        case 1: c.tile_w = 32; c.wp = 40; c.p = 16; c.ty = 12; c.rows = shape_row_spread(16, 0); break;
        case 2: c.tile_w = 64; c.wp = 72; c.p = 8; c.ty = 12; break;
        case 3: c.tile_w = 32; c.wp = 40; c.p = 8; c.ty = 16; c.rows = shape_row_spread(8, 0); break;
        case 4: c.tile_w = 32; c.wp = 40; c.p = 4; c.ty = 16; c.rows = shape_row_spread(4, 0); break;
        case 5:  // 32 x 16 with the shared maximum: 16 warps
            c.tile_w = 32; c.wp = 40; c.p = 16; c.ty = 16; c.merge = 1; c.rows = shape_row_spread(16, 1);
            c.smem_bytes -= 32 * 16 * 8;  // the keys sit ahead of the windows
            break;
        case 6:  // the same with 14 warps (146 registers a thread)
            c.tile_w = 32; c.wp = 40; c.p = 16; c.ty = 14; c.merge = 1; c.rows = shape_row_spread(16, 1);
            c.smem_bytes -= 32 * 16 * 8;
            break;
        case 7: c.tile_w = 32; c.wp = 40; c.p = 12; c.ty = 16; c.rows = shape_row_spread(12, 0); break;
        case 8:  // 32 x 20 with the shared maximum: 16 warps
            c.tile_w = 32; c.wp = 40; c.p = 20; c.ty = 16; c.merge = 1; c.rows = shape_row_spread(20, 1);
            c.smem_bytes -= 32 * 20 * 8;
            break;
        default: throw std::runtime_error("stack: unknown tile shape");
    }
    return c;
}

bool stack_shape_fits(const StackConfig& c, int n) {
    // the windows of all frames with 4 rows of vertical spread in at most 70 % of
    // shared memory (the rest: more spread and the offset table)
    const long long need = static_cast<long long>(n) * roundup(c.p + 4, c.bh) * c.wp * 4;
    return need <= static_cast<long long>(c.smem_bytes) * 7 / 10;
}

StackConfig choose_stack_config(int w, int h, int n, int smem_optin) {
    (void)w;
    (void)h;
    const int forced = g_shape;
    if (forced > 0) {
        const StackConfig c = stack_shape_config(forced, smem_optin);
        if (stack_shape_fits(c, n)) return c;
    }
    // the first shape whose windows fit: single-column tiles of 16, 8 and 4 rows
    // (taller frame stacks need the shorter tiles)
    for (int s : {1, 3}) {
        const StackConfig c = stack_shape_config(s, smem_optin);
        if (stack_shape_fits(c, n)) return c;
    }
    return stack_shape_config(4, smem_optin);
}

StackPlan make_stack_plan(int w, int h, int n, const int* dx, const int* dy, int m, int min_count,
                          const std::vector<int>& order, const StackConfig& cfg) {
    if (w <= 0 || h <= 0 || n <= 0 || m <= 0) throw std::runtime_error("stack pass: empty frames or motions");
    if (min_count < 1) throw std::runtime_error("stack pass: min_count must be at least 1");
    constexpr int M = kMotionBlock;
    if (cfg.mblock != M || order.size() % M != 0) throw std::runtime_error("stack plan: motions not in blocks");
    StackPlan P;
    P.w = w;
    P.h = h;
    P.n = n;
    P.m = m;
    P.min_count = min_count;
    P.pitch = frame_pitch(w);
    P.cfg = cfg;
    P.adds = static_cast<double>(m) * n * w * h;
    const int TW = cfg.tile_w, TH = cfg.tile_h(), WP = cfg.wp, BH = cfg.bh;
    // shared memory in floats after the barrier and alignment slack
    const long long budget = (cfg.smem_bytes - 256) / 4;

    P.inv_sqrt.assign(static_cast<size_t>(n) + 1, 0.0f);
    for (int c = 1; c <= n; ++c) P.inv_sqrt[static_cast<size_t>(c)] = static_cast<float>(1.0 / std::sqrt(static_cast<double>(c)));

    // clamped shifts: beyond +-w / +-h a frame never covers, as within
    auto cdx = [&](int j, int i) { return std::clamp(dx[static_cast<size_t>(j) * n + i], -w, w); };
    auto cdy = [&](int j, int i) { return std::clamp(dy[static_cast<size_t>(j) * n + i], -h, h); };
    for (size_t e = 0; e < order.size(); ++e) {
        if (order[e] >= m || (e % M == 0 && order[e] < 0))
            throw std::runtime_error("stack plan: motion blocks out of range or without motions");
    }
    // a block whose windows (the tile plus its motions' row spread, in every
    // frame) do not fit in shared memory on their own is split into single motions
    std::vector<int> blocks;
    blocks.reserve(order.size());
    for (size_t b = 0; b < order.size(); b += M) {
        long long rows = 0;
        int real = 0;
        bool fits = true;
        for (int k = 0; k < M; ++k) real += order[b + k] >= 0;
        for (int i = 0; i < n && real > 1; ++i) {
            int lx = INT32_MAX, hx = INT32_MIN, ly = INT32_MAX, hy = INT32_MIN;
            for (int k = 0; k < M; ++k) {
                const int j = order[b + k];
                if (j < 0) continue;
                lx = std::min(lx, cdx(j, i));
                hx = std::max(hx, cdx(j, i));
                ly = std::min(ly, cdy(j, i));
                hy = std::max(hy, cdy(j, i));
            }
            if (hx - floor4(lx) + TW > WP) fits = false;
            rows += roundup(TH + hy - ly, BH);
        }
        const long long table1 = std::max(static_cast<long long>(roundup(M * n, 8)) / 2,
                                          static_cast<long long>(roundup((n + 1) * 4, 16)) / 4);
        if (real > 1 && (!fits || rows * WP + table1 > budget)) {
            for (int k = 0; k < M; ++k)
                if (order[b + k] >= 0) blocks.insert(blocks.end(), {order[b + k], -1, -1, -1});
        } else if (real > 1 && cfg.rows > 0 && cfg.rows < kRowSpread) {
            // a kernel that takes smaller row offsets: consecutive runs of the
            // block whose rows stay within cfg.rows in every frame
            std::vector<int> run;
            std::vector<int> lo(static_cast<size_t>(n)), hi(static_cast<size_t>(n));
            auto close = [&]() {
                for (int k = 0; k < M; ++k) blocks.push_back(k < static_cast<int>(run.size()) ? run[static_cast<size_t>(k)] : -1);
                run.clear();
            };
            for (int k = 0; k < M; ++k) {
                const int j = order[b + k];
                if (j < 0) continue;
                bool ok = !run.empty();
                for (int i = 0; i < n && ok; ++i)
                    ok = std::max(hi[static_cast<size_t>(i)], cdy(j, i)) - std::min(lo[static_cast<size_t>(i)], cdy(j, i)) <=
                         cfg.rows;
                if (!ok && !run.empty()) close();
                if (run.empty())
                    for (int i = 0; i < n; ++i) lo[static_cast<size_t>(i)] = hi[static_cast<size_t>(i)] = cdy(j, i);
                for (int i = 0; i < n; ++i) {
                    lo[static_cast<size_t>(i)] = std::min(lo[static_cast<size_t>(i)], cdy(j, i));
                    hi[static_cast<size_t>(i)] = std::max(hi[static_cast<size_t>(i)], cdy(j, i));
                }
                run.push_back(j);
            }
            if (!run.empty()) close();
        } else {
            blocks.insert(blocks.end(), order.begin() + static_cast<long long>(b),
                          order.begin() + static_cast<long long>(b) + M);
        }
    }
    const int nblk = static_cast<int>(blocks.size()) / M;
    // each block's motions in ascending index, pads last: the kernel's in-block
    // maximum then keeps the first of equal S/N with a strict comparison
    for (int b = 0; b < nblk; ++b)
        std::sort(blocks.begin() + static_cast<long long>(b) * M, blocks.begin() + static_cast<long long>(b + 1) * M,
                  [](int a, int c) { return a >= 0 && (c < 0 || a < c); });
    // slot k of block b, pads standing for the block's last motion (their
    // windows and offsets repeat it; their slot_motion is -1)
    auto slot = [&](int b, int k) {
        int j = -1;
        for (int q = 0; q <= k; ++q)
            if (blocks[static_cast<size_t>(b) * M + q] >= 0) j = blocks[static_cast<size_t>(b) * M + q];
        return j;
    };

    std::vector<int> mnx(static_cast<size_t>(n)), mxx(static_cast<size_t>(n)), mny(static_cast<size_t>(n)),
        mxy(static_cast<size_t>(n));
    std::vector<int> tnx(mnx), txx(mxx), tny(mny), txy(mxy);
    std::vector<int> members;  // blocks of the open group

    // offset table of a group of `nb` blocks, in floats (the 16-bit slot table,
    // the larger of the two forms)
    // the larger of the two table forms: 16-bit slot offsets, or row descriptors
    // with their frame of zeros
    auto table_floats = [&](int nb) {
        return std::max(static_cast<long long>(roundup(nb * M * n, 8)) / 2,
                        static_cast<long long>(roundup(nb * (n + 1) * 4, 16)) / 4);
    };
    auto flush = [&]() {
        StackGroup g;
        g.slot0 = static_cast<int>(P.slot_motion.size());
        const int nb = static_cast<int>(members.size());
        g.nslots = nb * M;
        g.win0 = static_cast<int>(P.wins.size());
        g.gdxmin = g.gdymin = std::numeric_limits<int>::max();
        g.gdxmax = g.gdymax = std::numeric_limits<int>::min();
        int row = 0;
        for (int i = 0; i < n; ++i) {
            StackWin wv;
            wv.dx0 = floor4(mnx[static_cast<size_t>(i)]);
            wv.dy0 = mny[static_cast<size_t>(i)];
            wv.rows = roundup(TH + mxy[static_cast<size_t>(i)] - mny[static_cast<size_t>(i)], BH);
            wv.row0 = row;
            row += wv.rows;
            P.wins.push_back(wv);
            g.gdxmin = std::min(g.gdxmin, mnx[static_cast<size_t>(i)]);
            g.gdxmax = std::max(g.gdxmax, mxx[static_cast<size_t>(i)]);
            g.gdymin = std::min(g.gdymin, mny[static_cast<size_t>(i)]);
            g.gdymax = std::max(g.gdymax, mxy[static_cast<size_t>(i)]);
        }
        g.rows_total = row;
        // window offset of slot (q, k) in frame i
        auto offset = [&](int q, int k, int i) {
            const int j = slot(members[static_cast<size_t>(q)], k);
            const StackWin& wv = P.wins[static_cast<size_t>(g.win0 + i)];
            const long long off =
                static_cast<long long>(wv.row0 + cdy(j, i) - wv.dy0) * WP + (cdx(j, i) - wv.dx0);
            if (off < 0 || off > 65535) throw std::runtime_error("stack plan: window offset out of range");
            return static_cast<int>(off);
        };
        // row descriptors when every block shares its column in every frame
        bool fast = cfg.rows != 0;
        for (int q = 0; q < nb && fast; ++q)
            for (int i = 0; i < n && fast; ++i) {
                const int j0 = slot(members[static_cast<size_t>(q)], 0);
                int lo = cdy(j0, i), hi = lo;
                for (int k = 1; k < M && fast; ++k) {
                    const int j = slot(members[static_cast<size_t>(q)], k);
                    fast = cdx(j, i) == cdx(j0, i);
                    lo = std::min(lo, cdy(j, i));
                    hi = std::max(hi, cdy(j, i));
                }
                fast = fast && hi - lo <= cfg.rows;
            }
        g.rows_fast = fast ? 1 : 0;
        // a row descriptor table holds one more frame of zeros: the kernel loads
        // frame i + 1's words while it adds frame i's
        g.tab_bytes = fast ? roundup(nb * (n + 1) * 4, 16) : roundup(g.nslots * n * 2, 16);
        P.max_rows = std::max(P.max_rows, row);
        P.max_group_bytes = std::max(P.max_group_bytes, static_cast<long long>(row) * WP * 4 + g.tab_bytes);
        P.max_slots = std::max(P.max_slots, g.nslots);
        P.slot_off_base.push_back(static_cast<int>(P.slot_off.size()));
        const size_t base = P.slot_off.size();
        P.slot_off.resize(base + static_cast<size_t>(g.tab_bytes) / 2, 0);
        if (fast) {
            // [frame][block] descriptors: lowest row's offset, each slot's row above it
            for (int i = 0; i < n; ++i)
                for (int q = 0; q < nb; ++q) {
                    int o[M];
                    int omin = 1 << 30;
                    for (int k = 0; k < M; ++k) {
                        o[k] = offset(q, k, i);
                        omin = std::min(omin, o[k]);
                    }
                    uint32_t d = static_cast<uint32_t>(omin), smax = 0;
                    for (int k = 0; k < M; ++k) {
                        const uint32_t dk = static_cast<uint32_t>((o[k] - omin) / WP);
                        d |= dk << (16 + 2 * k);
                        smax = std::max(smax, dk);
                    }
                    d |= smax << 24;
                    if (smax <= 1u)  // each slot's offset as one bit of a 4-bit pattern
                        for (int k = 0; k < M; ++k) d |= ((d >> (16 + 2 * k)) & 1u) << (26 + k);
                    const size_t e = base + 2 * (static_cast<size_t>(i) * nb + static_cast<size_t>(q));
                    P.slot_off[e] = static_cast<uint16_t>(d & 0xffffu);
                    P.slot_off[e + 1] = static_cast<uint16_t>(d >> 16);
                }
        } else {
            // [frame][slot] 16-bit offsets
            for (int q = 0; q < nb; ++q)
                for (int k = 0; k < M; ++k)
                    for (int i = 0; i < n; ++i)
                        P.slot_off[base + static_cast<size_t>(i) * g.nslots + static_cast<size_t>(q * M + k)] =
                            static_cast<uint16_t>(offset(q, k, i));
        }
        for (int q = 0; q < nb; ++q)
            for (int k = 0; k < M; ++k) {
                const int b = members[static_cast<size_t>(q)];
                P.slot_motion.push_back(blocks[static_cast<size_t>(b) * M + k]);
                const int j = slot(b, k);
                for (int i = 0; i < n; ++i)
                    P.slot_shift.push_back(make_short2(static_cast<short>(cdx(j, i)), static_cast<short>(cdy(j, i))));
            }
        P.groups.push_back(g);
        members.clear();
    };

    // the bounds of the open group extended by block b (into tnx..txy); false
    // when its windows would not fit
    auto extend = [&](int b) {
        long long rows = 0;
        bool fits = true;
        for (int i = 0; i < n && fits; ++i) {
            const size_t k = static_cast<size_t>(i);
            int lx = members.empty() ? INT32_MAX : mnx[k], hx = members.empty() ? INT32_MIN : mxx[k];
            int ly = members.empty() ? INT32_MAX : mny[k], hy = members.empty() ? INT32_MIN : mxy[k];
            for (int q = 0; q < M; ++q) {
                const int j = blocks[static_cast<size_t>(b) * M + q];
                if (j < 0) continue;
                lx = std::min(lx, cdx(j, i));
                hx = std::max(hx, cdx(j, i));
                ly = std::min(ly, cdy(j, i));
                hy = std::max(hy, cdy(j, i));
            }
            tnx[k] = lx;
            txx[k] = hx;
            tny[k] = ly;
            txy[k] = hy;
            if (hx - floor4(lx) + TW > WP) fits = false;
            rows += roundup(TH + hy - ly, BH);
        }
        const int nb = static_cast<int>(members.size()) + 1;
        return fits && rows * WP + table_floats(nb) <= budget;
    };
    auto accept = [&](int b) {
        mnx.swap(tnx);
        mxx.swap(txx);
        mny.swap(tny);
        mxy.swap(txy);
        members.push_back(b);
    };
    auto start_group = [&](int b) {
        if (!extend(b)) throw std::runtime_error("stack plan: one motion block's frame windows exceed shared memory");
        accept(b);
    };
    auto recompute = [&]() {
        std::vector<int> keep;
        keep.swap(members);
        for (int b : keep) {
            extend(b);
            accept(b);
        }
    };
    std::function<void(int)> add_or_flush = [&](int b) {
        if (members.empty()) {
            start_group(b);
        } else if (extend(b)) {
            accept(b);
        } else {
            flush();
            start_group(b);
        }
    };
    for (int b = 0; b < nblk; ++b) {
        if (members.empty()) {
            start_group(b);
            continue;
        }
        if (extend(b)) {
            accept(b);
            continue;
        }
        // a full group: keep a whole number of blocks for every warp and carry
        // the rest into the next group
        const int share = cfg.ty;
        const int keep = static_cast<int>(members.size()) / share * share;
        std::vector<int> carry;
        if (keep > 0 && keep < static_cast<int>(members.size())) {
            carry.assign(members.begin() + keep, members.end());
            members.resize(static_cast<size_t>(keep));
            recompute();
        }
        flush();
        for (int c : carry) add_or_flush(c);
        add_or_flush(b);
    }
    if (!members.empty()) flush();
    return P;
}

void StackPlanDev::upload(const StackPlan& p, cudaStream_t s) {
    release();
    auto put = [&](auto*& dst, const auto& v) {
        using T = std::remove_reference_t<decltype(v[0])>;
        const size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
        FTB_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&dst), bytes, s));
        if (!v.empty()) FTB_CHECK(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    };
    put(groups, p.groups);
    put(wins, p.wins);
    put(slot_motion, p.slot_motion);
    put(slot_off, p.slot_off);
    put(slot_off_base, p.slot_off_base);
    put(slot_shift, p.slot_shift);
    put(inv_sqrt, p.inv_sqrt);
    ngroups = static_cast<int>(p.groups.size());
    stream_ = s;
}

void StackPlanDev::release() {
    for (void* q : {static_cast<void*>(groups), static_cast<void*>(wins), static_cast<void*>(slot_motion),
                    static_cast<void*>(slot_off), static_cast<void*>(slot_off_base), static_cast<void*>(slot_shift),
                    static_cast<void*>(inv_sqrt)})
        if (q) cudaFreeAsync(q, stream_);
    groups = nullptr;
    wins = nullptr;
    slot_motion = nullptr;
    slot_off = nullptr;
    slot_off_base = nullptr;
    slot_shift = nullptr;
    inv_sqrt = nullptr;
    ngroups = 0;
}

// ------------------------------------------------------------------ device

namespace {

struct StackArgs {
    int w, h, n, min_count;
    int g0, g1, first, last;
    int tiles_x, tiles_y;  // tile grid of this pass (tiles_y: rows of it in this launch)
    int ty0;               // first tile row
    long long item0;       // its first work item in the batch
    const StackGroup* groups;
    const StackWin* wins;
    const int* slot_motion;
    const uint16_t* slot_off;
    const int* slot_off_base;
    const short2* slot_shift;
    const float* inv_sqrt;
    float* best;
    int* arg;
    float* max_snr;
    int* best_v;
    int* err;
    unsigned extra_tx;      // bytes the staging barrier expects beyond its copies (0; a test of the bounded wait)
    long long wait_limit;   // clock cycles a staging wait may take
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bounded wait on the staging barrier: `limit` clock cycles (about two seconds
// by default), then the kernel records an error and gives up (the host turns it
// into an exception).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, long long limit) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit) {
            atomicExch(err, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

template <int P, int WP>
__device__ __forceinline__ void load_column(float (&v)[P], const float* __restrict__ src) {
#pragma unroll
    for (int p = 0; p < P; ++p) v[p] = src[p * WP];
}

template <int P>
__device__ __forceinline__ void add_column(float (&acc)[P], const float (&v)[P]) {
#pragma unroll
    for (int p = 0; p < P; ++p) acc[p] = __fadd_rn(acc[p], v[p]);
}

// The four slot offsets of a block for frame i, from the group's [frame][slot]
// table of 16-bit window offsets.
__device__ __forceinline__ uint2 block_offsets(const uint16_t* __restrict__ offs, const StackGroup& G, int s0, int i) {
    return *reinterpret_cast<const uint2*>(offs + i * G.nslots + s0);
}

// The maximum of one block's motions at one pixel. A block's slots hold its
// motions in ascending index with pads repeating the last one, so a strict
// comparison keeps the first of equal S/N and a pad (equal to the slot before
// it) never wins; starting from -inf with no motion, NaN and -inf never enter.
__device__ __forceinline__ void block_max(float s, int j, float& b, int& bj) {
    if (s > b) {
        b = s;
        bj = j;
    }
}

// The block's maximum into the running one: larger S/N, and of equal S/N the
// smaller motion index (backend_cpu.cpp:77-204). A block maximum of -inf has no
// motion (-1) and then changes nothing: a running -inf also has none.
__device__ __forceinline__ void merge_max(float b, int bj, float& best, int& arg) {
    if (b > best || (b == best && bj < arg)) {
        best = b;
        arg = bj;
    }
}

// One block of 4 consecutive motions of a group for this thread's P pixels
// (one column, P rows), frames in ascending order. A motion whose window offset
// for frame i equals the previous motion's adds the P values already in
// registers instead of loading them again; the offsets are the same for the
// whole CTA, so these branches are warp-uniform.
// BORDER: coverage counts. A frame that covers the whole tile for a motion (the
// common case; a warp-uniform test) adds 1 to the motion's count, a frame that
// covers part of it is counted per pixel (8-bit counters, 4 per register).
template <int P, int WP, bool BORDER>
__device__ __forceinline__ void motion_quad(const StackArgs& a, const StackGroup& G, int s0,
                                            const float* __restrict__ win, const uint16_t* __restrict__ offs, int tb,
                                            int x, int x0, int y0, float inv_n, float (&best)[P], int (&arg)[P]) {
    constexpr int M = 4;
    constexpr int PW = (P + 3) / 4;
    float acc[M][P];
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int p = 0; p < P; ++p) acc[k][p] = 0.0f;
    int cfull[M] = {0, 0, 0, 0};
    uint32_t cpart[M][PW];
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int w = 0; w < PW; ++w) cpart[k][w] = 0;
    // the next frame's four offsets are loaded one frame ahead, so the reuse
    // tests below do not wait on a shared-memory load
    const int n = a.n;  // loop bounds and table strides in registers, not reloaded from the pass arguments
    uint2 qn = block_offsets(offs, G, s0, 0);
    for (int i = 0; i < n; ++i) {
        const uint2 q = qn;
        if (i + 1 < n) qn = block_offsets(offs, G, s0, i + 1);
        const uint32_t o0 = q.x & 0xffffu, o1 = q.x >> 16, o2 = q.y & 0xffffu, o3 = q.y >> 16;
        float v[P];
        load_column<P, WP>(v, win + o0 + tb);
        add_column<P>(acc[0], v);
        if (o1 != o0) load_column<P, WP>(v, win + o1 + tb);
        add_column<P>(acc[1], v);
        if (o2 != o1) load_column<P, WP>(v, win + o2 + tb);
        add_column<P>(acc[2], v);
        if (o3 != o2) load_column<P, WP>(v, win + o3 + tb);
        add_column<P>(acc[3], v);
        if constexpr (BORDER) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const short2 sh = a.slot_shift[static_cast<size_t>(G.slot0 + s0 + k) * n + i];
                const bool whole = x0 + sh.x >= 0 && x0 + 31 + sh.x < a.w && y0 + sh.y >= 0 && y0 + P - 1 + sh.y < a.h;
                if (whole) {
                    ++cfull[k];
                } else {
                    const bool inx = static_cast<unsigned>(x + sh.x) < static_cast<unsigned>(a.w);
#pragma unroll
                    for (int p = 0; p < P; ++p)
                        if (inx && static_cast<unsigned>(y0 + p + sh.y) < static_cast<unsigned>(a.h))
                            cpart[k][p / 4] += 1u << (8 * (p % 4));
                }
            }
        }
    }
    if constexpr (!BORDER) {
        int jk[M];
#pragma unroll
        for (int k = 0; k < M; ++k) jk[k] = a.slot_motion[G.slot0 + s0 + k];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            float b = -CUDART_INF_F;
            int bj = -1;
#pragma unroll
            for (int k = 0; k < M; ++k) block_max(__fmul_rn(acc[k][p], inv_n), jk[k], b, bj);
            merge_max(b, bj, best[p], arg[p]);
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < M; ++k) {
        const int j = a.slot_motion[G.slot0 + s0 + k];
        if (j < 0) continue;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            float f = inv_n;
            if constexpr (BORDER) {
                const int c = cfull[k] + static_cast<int>((cpart[k][p / 4] >> (8 * (p % 4))) & 0xffu);
                if (c < a.min_count) continue;
                f = a.inv_sqrt[c];
            }
            const float s = __fmul_rn(acc[k][p], f);
            if (s > best[p] || (s == best[p] && j < arg[p])) {
                best[p] = s;
                arg[p] = j;
            }
        }
    }
}

// ---- one shared maximum per tile: instead of a best/argmax pair per pixel in
// every thread, the CTA's warps merge into one array of 64-bit keys in shared
// memory with atomicMax. key = (order-preserving bits of S/N) << 32 | ~index,
// so a larger S/N wins and equal S/N goes to the lower motion index -- the
// reference's rule. S/N is never -0.0 (sums start at +0.0f and round to
// nearest) and -inf / NaN never enter, as in the register rule. Frees 2P
// registers per thread, so 16-row tiles run 16 warps.

__device__ __forceinline__ unsigned long long snr_key(float s, int j) {
    const uint32_t b = __float_as_uint(s);
    const uint32_t o = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return (static_cast<unsigned long long>(o) << 32) | static_cast<uint32_t>(~j);
}

__device__ __forceinline__ void snr_unkey(unsigned long long k, float& s, int& j) {
    const uint32_t o = static_cast<uint32_t>(k >> 32);
    s = __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
    j = static_cast<int>(~static_cast<uint32_t>(k));
}

// Pairs of floats: __fadd2_rn / __fmul2_rn are two independent
// round-to-nearest operations per call, bit-identical to two scalar ones
// (__fadd_rn / __fmul_rn), issued as one paired instruction on sm_100.
// The adds of one frame for a block whose motions sit 0 or 1 row above the
// block's base: bit k of PT is motion k's row offset.
template <int PT, int H>
__device__ __forceinline__ void add_pattern(float2 (&acc)[4][H], const float2* A) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int dk = (PT >> k) & 1;  // a constant once the loop is unrolled
#pragma unroll
        for (int q = 0; q < H; ++q) acc[k][q] = __fadd2_rn(acc[k][q], A[q + dk]);
    }
}

// Coverage of a border tile's pixels by a block's motions: cx counts the frames
// whose rows cover the whole tile for every motion and whose column covers
// this thread's pixels; cpart[k] holds, one byte a row, the frames that cover
// row p of motion k's pixels otherwise. A pixel's frame count is cx plus its
// byte (frames never exceed 255).
template <int P>
struct BorderCount {
    static constexpr int PW = (P + 3) / 4;
    int cx = 0;
    uint32_t cpart[4][PW] = {};
    __device__ __forceinline__ int count(int k, int p) const {
        return cx + static_cast<int>((cpart[k][p >> 2] >> (8 * (p & 3))) & 0xffu);
    }
};

// One block of 4 motions of a rows_fast group for this thread's P pixels (one
// column, P rows), frames in ascending order. In every frame the block's
// motions read one column of the window at row offsets 0..3 above the
// descriptor's base, so the thread loads that column once (P + S rows, S = the
// largest row offset) and every motion adds its P rows from registers. Rows are
// paired across the two halves of the tile, row q with row q + P/2, and each
// pair is one add.rn.f32x2: register pair A[r] holds rows (r, r + P/2), so
// motion k adds A[q + row offset] to its accumulator pair q (rows P/2 .. P/2 +
// S - 1 are loaded twice, once for each pairing). Outside the frame the windows
// hold +0.0f (the copies' zero fill), which adds nothing to a sum that starts
// at +0.0f, so the sums of a border tile are the reference's truncated sums;
// with COUNT the frames covering each pixel are counted as well, from the
// block's first slot's shift and the descriptor's row offsets.
template <int P, int WP, int SMAX, bool COUNT>
__device__ __forceinline__ void rows_accumulate(const StackArgs& a, const StackGroup& G, int s0,
                                                const float* __restrict__ win, const uint16_t* __restrict__ offs,
                                                int tb, float2 (&acc)[4][P / 2], int x, int y0,
                                                BorderCount<P>& cov) {
    constexpr int M = 4;
    constexpr int H = P / 2;
    static_assert(P % 2 == 0, "rows are paired");
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int q = 0; q < H; ++q) acc[k][q] = make_float2(0.0f, 0.0f);
    const int n = a.n, nb = G.nslots >> 2;
    const uint32_t* dp = reinterpret_cast<const uint32_t*>(offs) + (s0 >> 2);
    // the descriptor is the same word in every lane; the broadcast from lane 0
    // lets the compiler treat it, and the branches on it, as warp-uniform
    uint32_t dn = __shfl_sync(0xffffffffu, dp[0], 0);
    for (int i = 0; i < n; ++i) {
        const uint32_t d = dn;
        // the table's extra frame makes the last prefetch a zero word
        dn = __shfl_sync(0xffffffffu, dp[(i + 1) * nb], 0);
        const float* src = win + (d & 0xffffu) + tb;
        float2 A[H + SMAX];
#pragma unroll
        for (int r = 0; r < H; ++r) A[r] = make_float2(src[r * WP], src[(r + H) * WP]);
        if constexpr (COUNT) {
            const short2 sh = a.slot_shift[static_cast<size_t>(G.slot0 + s0) * n + i];
            const int dylow = sh.y - static_cast<int>((d >> 16) & 3u), smax = static_cast<int>((d >> 24) & 3u);
            const bool inx = static_cast<unsigned>(x + sh.x) < static_cast<unsigned>(a.w);
            if (y0 + dylow >= 0 && y0 + P - 1 + dylow + smax < a.h) {
                cov.cx += inx ? 1 : 0;
            } else if (inx) {
#pragma unroll
                for (int k = 0; k < M; ++k) {
                    const int dy = dylow + static_cast<int>((d >> (16 + 2 * k)) & 3u);
                    const int lo = max(0, -(y0 + dy)), hi = min(P - 1, a.h - 1 - (y0 + dy));
                    if (lo > hi) continue;
                    // rows lo..hi as bits, then each row's bit as one byte of its word
                    const uint32_t m = (0xffffffffu >> (31 - hi)) & (0xffffffffu << lo);
#pragma unroll
                    for (int w = 0; w < BorderCount<P>::PW; ++w)
                        cov.cpart[k][w] += (((m >> (4 * w)) & 15u) * 0x00204081u) & 0x01010101u;
                }
            }
        }
        if (d < (1u << 24)) {
            // every motion on the base row (no row offset, pattern 0): the most
            // common frame of a block, tested first
#pragma unroll
            for (int k = 0; k < M; ++k)
#pragma unroll
                for (int q = 0; q < H; ++q) acc[k][q] = __fadd2_rn(acc[k][q], A[q]);
            continue;
        }
        const uint32_t S = (d >> 24) & 3u;
        if (S >= 1u) A[H] = make_float2(src[H * WP], src[P * WP]);
        if (S <= 1u) {
            // row offsets 0 or 1: one branch on the block's 4-bit pattern, each
            // case a straight run of adds with fixed register pairs
            switch ((d >> 26) & 15u) {
#define FTB_PATTERN_CASE(PT) \
    case PT:                 \
        add_pattern<PT, H>(acc, A); \
        break;
                FTB_PATTERN_CASE(0) FTB_PATTERN_CASE(1) FTB_PATTERN_CASE(2) FTB_PATTERN_CASE(3)
                FTB_PATTERN_CASE(4) FTB_PATTERN_CASE(5) FTB_PATTERN_CASE(6) FTB_PATTERN_CASE(7)
                FTB_PATTERN_CASE(8) FTB_PATTERN_CASE(9) FTB_PATTERN_CASE(10) FTB_PATTERN_CASE(11)
                FTB_PATTERN_CASE(12) FTB_PATTERN_CASE(13) FTB_PATTERN_CASE(14) FTB_PATTERN_CASE(15)
#undef FTB_PATTERN_CASE
            }
            continue;
        }
        if constexpr (SMAX >= 3) {  // row offsets up to 3 (the planner keeps SMAX)
        if (S >= 2u) A[H + 1] = make_float2(src[(H + 1) * WP], src[(P + 1) * WP]);
        if (S >= 3u) A[H + 2] = make_float2(src[(H + 2) * WP], src[(P + 2) * WP]);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const uint32_t dk = (d >> (16 + 2 * k)) & 3u;
            if (dk == 0u) {
#pragma unroll
                for (int q = 0; q < H; ++q) acc[k][q] = __fadd2_rn(acc[k][q], A[q]);
            } else if (dk == 1u) {
#pragma unroll
                for (int q = 0; q < H; ++q) acc[k][q] = __fadd2_rn(acc[k][q], A[q + 1]);
            } else if (dk == 2u) {
#pragma unroll
                for (int q = 0; q < H; ++q) acc[k][q] = __fadd2_rn(acc[k][q], A[q + 2]);
            } else {
#pragma unroll
                for (int q = 0; q < H; ++q) acc[k][q] = __fadd2_rn(acc[k][q], A[q + 3]);
            }
        }
        }
    }
}

// The block's maxima at row pairs (q, q + P/2) from the row-paired sums.
template <int P>
__device__ __forceinline__ void rows_block_max(const float2 (&acc)[4][P / 2], const int (&jk)[4], float inv_n, int q,
                                               float& bl, int& al, float& bh, int& ah) {
    const float2 inv2 = make_float2(inv_n, inv_n);
    bl = bh = -CUDART_INF_F;
    al = ah = -1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 sn = __fmul2_rn(acc[k][q], inv2);
        block_max(sn.x, jk[k], bl, al);
        block_max(sn.y, jk[k], bh, ah);
    }
}

// rows_accumulate for one block, its maxima into this thread's running ones.
template <int P, int WP, int SMAX>
__device__ __forceinline__ void motion_quad_rows(const StackArgs& a, const StackGroup& G, int s0,
                                                 const float* __restrict__ win, const uint16_t* __restrict__ offs,
                                                 int tb, float inv_n, float (&best)[P], int (&arg)[P]) {
    constexpr int H = P / 2;
    float2 acc[4][H];
    BorderCount<P> cov;
    rows_accumulate<P, WP, SMAX, false>(a, G, s0, win, offs, tb, acc, 0, 0, cov);
    int jk[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) jk[k] = a.slot_motion[G.slot0 + s0 + k];
#pragma unroll
    for (int q = 0; q < H; ++q) {
        float bl, bh;
        int al, ah;
        rows_block_max<P>(acc, jk, inv_n, q, bl, al, bh, ah);
        merge_max(bl, al, best[q], arg[q]);
        merge_max(bh, ah, best[q + H], arg[q + H]);
    }
}

// The block's maximum at pixel row p of a border tile: each motion's sum times
// 1 / sqrt(frames covering the pixel), motions covered by fewer than min_count
// frames left out (backend_cpu.cpp:77-204).
template <int P>
__device__ __forceinline__ void border_block_max(const StackArgs& a, const float2 (&acc)[4][P / 2],
                                                 const BorderCount<P>& cov, const int (&jk)[4], int p, float& b,
                                                 int& bj) {
    constexpr int H = P / 2;
    b = -CUDART_INF_F;
    bj = -1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = cov.count(k, p);
        if (c < a.min_count) continue;
        const float sum = p < H ? acc[k][p].x : acc[k][p - H].y;
        block_max(__fmul_rn(sum, a.inv_sqrt[c]), jk[k], b, bj);
    }
}

// The same block on a border tile: sums by the row-descriptor path, the frames
// covering each pixel counted beside them.
template <int P, int WP, int SMAX>
__device__ __forceinline__ void motion_quad_rows_border(const StackArgs& a, const StackGroup& G, int s0,
                                                        const float* __restrict__ win,
                                                        const uint16_t* __restrict__ offs, int tb, int x, int y0,
                                                        float (&best)[P], int (&arg)[P]) {
    float2 acc[4][P / 2];
    BorderCount<P> cov;
    rows_accumulate<P, WP, SMAX, true>(a, G, s0, win, offs, tb, acc, x, y0, cov);
    int jk[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) jk[k] = a.slot_motion[G.slot0 + s0 + k];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float b;
        int bj;
        border_block_max<P>(a, acc, cov, jk, p, b, bj);
        merge_max(b, bj, best[p], arg[p]);
    }
}

// rows_accumulate for one block, its maxima into the tile's shared keys (one
// atomic per pixel that has a motion: a block maximum above -inf).
template <int P, int WP, int SMAX>
__device__ __forceinline__ void motion_quad_rows_atom(const StackArgs& a, const StackGroup& G, int s0,
                                                      const float* __restrict__ win,
                                                      const uint16_t* __restrict__ offs, int tb, float inv_n,
                                                      unsigned long long* keys) {
    constexpr int H = P / 2;
    float2 acc[4][H];
    BorderCount<P> cov;
    rows_accumulate<P, WP, SMAX, false>(a, G, s0, win, offs, tb, acc, 0, 0, cov);
    int jk[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) jk[k] = a.slot_motion[G.slot0 + s0 + k];
#pragma unroll
    for (int q = 0; q < H; ++q) {
        float bl, bh;
        int al, ah;
        rows_block_max<P>(acc, jk, inv_n, q, bl, al, bh, ah);
        if (al >= 0) atomicMax(keys + q * 32 + tb, snr_key(bl, al));
        if (ah >= 0) atomicMax(keys + (q + H) * 32 + tb, snr_key(bh, ah));
    }
}

// The same on a border tile, into the shared keys.
template <int P, int WP, int SMAX>
__device__ __forceinline__ void motion_quad_rows_border_atom(const StackArgs& a, const StackGroup& G, int s0,
                                                             const float* __restrict__ win,
                                                             const uint16_t* __restrict__ offs, int tb, int x, int y0,
                                                             unsigned long long* keys) {
    float2 acc[4][P / 2];
    BorderCount<P> cov;
    rows_accumulate<P, WP, SMAX, true>(a, G, s0, win, offs, tb, acc, x, y0, cov);
    int jk[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) jk[k] = a.slot_motion[G.slot0 + s0 + k];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        float b;
        int bj;
        border_block_max<P>(a, acc, cov, jk, p, b, bj);
        if (bj >= 0) atomicMax(keys + p * 32 + tb, snr_key(b, bj));
    }
}

// Stages group g for the tile at (x0, y0): every frame's window by TMA (the
// lanes of warp 0 share the copies) and the group's 16-bit offset table by one
// bulk copy, all completing on the one mbarrier; resets the block counter the
// warps take 4-motion blocks from. Returns false if the staging wait timed out
// (every thread then returns; the host reports the error).
template <int NW, int WP, int BH>
__device__ __forceinline__ bool stage_group(const StackArgs& a, const StackGroup& G, int g, const CUtensorMap* tmap,
                                            int x0, int y0, uint64_t* bar, float* win, uint16_t* offs, int* block_next,
                                            int* err, uint32_t& phase) {
    const int tid = threadIdx.x, lane = tid & 31;
    // the previous group's windows and offsets are no longer read, and this
    // thread's generic-proxy stores are ordered before the async writes below
    fence_proxy_async();
    __syncthreads();
    if (tid < 32) {
        const uint32_t tab_bytes = static_cast<uint32_t>(G.tab_bytes);
        if (lane == 0) {
            *block_next = NW;  // blocks 0 .. NW-1 go to the warps in order
            mbar_expect_tx(bar, static_cast<uint32_t>(G.rows_total * WP * 4) + tab_bytes + a.extra_tx);
        }
        __syncwarp();
        if (lane == 0) bulk_load(offs, a.slot_off + a.slot_off_base[g], tab_bytes, bar);
        for (int i = lane; i < a.n; i += 32) {
            const StackWin wv = a.wins[G.win0 + i];
            for (int b = 0; b < wv.rows; b += BH)
                tma_load_3d(win + (wv.row0 + b) * WP, tmap, x0 + wv.dx0, y0 + wv.dy0 + b, i, bar);
        }
    }
    const bool ok = mbar_wait_bounded(bar, phase, err, a.wait_limit);
    if (__syncthreads_or(!ok)) return false;
    phase ^= 1u;
    return true;
}

// The next 4-motion block for this warp from the group's counter.
__device__ __forceinline__ int next_block(int* block_next) {
    int q = 0;
    if ((threadIdx.x & 31) == 0) q = atomicAdd(block_next, 1);
    return __shfl_sync(0xffffffffu, q, 0);
}

// One 32 x P output tile of one pass: the CTA's NW warps share the tile and
// split each group's 4-motion blocks; per-warp maxima merge through shared memory
// at the end. Returns false if a staging wait timed out.
template <int NW, int P, int WP, int BH>
__device__ bool stack_tile(const StackArgs& a, const CUtensorMap* tmap, int x0, int y0, uint64_t* bar, float* win,
                           int* block_next, int* err, uint32_t& phase) {
    constexpr int M = 4;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x = x0 + lane;
    const int tb = lane;  // thread's first window element relative to a motion's offset

    float best[P];
    int arg[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        best[p] = -CUDART_INF_F;
        arg[p] = -1;
    }
    const bool full = x0 + 31 < a.w && y0 + P - 1 < a.h;
    const float inv_n = a.inv_sqrt[a.n];
    for (int g = a.g0; g < a.g1; ++g) {
        const StackGroup G = a.groups[g];
        uint16_t* offs = reinterpret_cast<uint16_t*>(win + G.rows_total * WP);
        if (!stage_group<NW, WP, BH>(a, G, g, tmap, x0, y0, bar, win, offs, block_next, err, phase)) return false;
        const bool interior = full && x0 + G.gdxmin >= 0 && x0 + 31 + G.gdxmax < a.w && y0 + G.gdymin >= 0 &&
                              y0 + P - 1 + G.gdymax < a.h;
        // blocks by a shared counter: a warp whose blocks reuse more loads takes more of them
        if (G.rows_fast) {
            if (interior) {
                for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                    motion_quad_rows<P, WP, shape_row_spread(P, 0)>(a, G, s0, win, offs, tb, inv_n, best, arg);
            } else {
                for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                    motion_quad_rows_border<P, WP, shape_row_spread(P, 0)>(a, G, s0, win, offs, tb, x, y0, best, arg);
            }
        } else if (interior) {
            for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                motion_quad<P, WP, false>(a, G, s0, win, offs, tb, x, x0, y0, inv_n, best, arg);
        } else {
            for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                motion_quad<P, WP, true>(a, G, s0, win, offs, tb, x, x0, y0, inv_n, best, arg);
        }
    }
    // merge the warps' maxima (and, for a continued pass, the stored running ones)
    __syncthreads();
    float* mb = win;
    int* ma = reinterpret_cast<int*>(win + NW * 32 * P);
#pragma unroll
    for (int p = 0; p < P; ++p) {
        mb[(warp * P + p) * 32 + lane] = best[p];
        ma[(warp * P + p) * 32 + lane] = arg[p];
    }
    __syncthreads();
    for (int q = tid; q < 32 * P; q += 32 * NW) {
        const int p = q >> 5, l = q & 31;
        const int xx = x0 + l, yy = y0 + p;
        if (xx >= a.w || yy >= a.h) continue;
        const size_t o = static_cast<size_t>(yy) * a.w + xx;
        float b = -CUDART_INF_F;
        int ar = -1;
        if (!a.first) {
            b = a.best[o];
            ar = a.arg[o];
        }
        for (int w = 0; w < NW; ++w) {
            const float s = mb[(w * P + p) * 32 + l];
            const int j = ma[(w * P + p) * 32 + l];
            if (j >= 0 && (s > b || (s == b && (ar < 0 || j < ar)))) {
                b = s;
                ar = j;
            }
        }
        if (a.last) {
            a.max_snr[o] = isfinite(b) ? b : 0.0f;
            a.best_v[o] = ar;
        } else {
            a.best[o] = b;
            a.arg[o] = ar;
        }
    }
    __syncthreads();  // the merge area is reused by the next tile's windows
    return true;
}

template <int P, int WP, bool BORDER>
__device__ __forceinline__ void motion_quad_atom(const StackArgs& a, const StackGroup& G, int s0,
                                                 const float* __restrict__ win, const uint16_t* __restrict__ offs,
                                                 int tb, int x, int x0, int y0, float inv_n, unsigned long long* keys) {
    constexpr int M = 4;
    constexpr int PW = (P + 3) / 4;
    float acc[M][P];
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int p = 0; p < P; ++p) acc[k][p] = 0.0f;
    int cfull[M] = {0, 0, 0, 0};
    uint32_t cpart[M][PW];
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int w = 0; w < PW; ++w) cpart[k][w] = 0;
    const int n = a.n;
    uint2 qn = block_offsets(offs, G, s0, 0);
    for (int i = 0; i < n; ++i) {
        const uint2 q = qn;
        if (i + 1 < n) qn = block_offsets(offs, G, s0, i + 1);
        const uint32_t o0 = q.x & 0xffffu, o1 = q.x >> 16, o2 = q.y & 0xffffu, o3 = q.y >> 16;
        float v[P];
        load_column<P, WP>(v, win + o0 + tb);
        add_column<P>(acc[0], v);
        if (o1 != o0) load_column<P, WP>(v, win + o1 + tb);
        add_column<P>(acc[1], v);
        if (o2 != o1) load_column<P, WP>(v, win + o2 + tb);
        add_column<P>(acc[2], v);
        if (o3 != o2) load_column<P, WP>(v, win + o3 + tb);
        add_column<P>(acc[3], v);
        if constexpr (BORDER) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const short2 sh = a.slot_shift[static_cast<size_t>(G.slot0 + s0 + k) * n + i];
                const bool whole = x0 + sh.x >= 0 && x0 + 31 + sh.x < a.w && y0 + sh.y >= 0 && y0 + P - 1 + sh.y < a.h;
                if (whole) {
                    ++cfull[k];
                } else {
                    const bool inx = static_cast<unsigned>(x + sh.x) < static_cast<unsigned>(a.w);
#pragma unroll
                    for (int p = 0; p < P; ++p)
                        if (inx && static_cast<unsigned>(y0 + p + sh.y) < static_cast<unsigned>(a.h))
                            cpart[k][p / 4] += 1u << (8 * (p % 4));
                }
            }
        }
    }
    int js[M];
#pragma unroll
    for (int k = 0; k < M; ++k) js[k] = a.slot_motion[G.slot0 + s0 + k];
#pragma unroll
    for (int p = 0; p < P; ++p) {
        // the block's best for this pixel, then one atomic
        float bs = -CUDART_INF_F;
        int bj = -1;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (js[k] < 0) continue;
            float f = inv_n;
            if constexpr (BORDER) {
                const int c = cfull[k] + static_cast<int>((cpart[k][p / 4] >> (8 * (p % 4))) & 0xffu);
                if (c < a.min_count) continue;
                f = a.inv_sqrt[c];
            }
            const float sv = __fmul_rn(acc[k][p], f);
            if (sv > bs || (sv == bs && bj >= 0 && js[k] < bj)) {
                bs = sv;
                bj = js[k];
            }
        }
        if (bj >= 0 && bs > -CUDART_INF_F) atomicMax(keys + p * 32 + (tb & 31), snr_key(bs, bj));
    }
}

// One 32 x P output tile with the shared maximum (as stack_tile otherwise).
template <int NW, int P, int WP, int BH>
__device__ bool stack_tile_atom(const StackArgs& a, const CUtensorMap* tmap, int x0, int y0, uint64_t* bar,
                                unsigned long long* keys, float* win, int* block_next, int* err, uint32_t& phase) {
    constexpr int M = 4;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x = x0 + lane;
    const int tb = lane;
    // the tile's running maximum: empty, or the stored one of a continued pass
    for (int q = tid; q < 32 * P; q += 32 * NW) {
        unsigned long long k = 0ull;
        const int xx = x0 + (q & 31), yy = y0 + (q >> 5);
        if (!a.first && xx < a.w && yy < a.h) {
            const size_t o = static_cast<size_t>(yy) * a.w + xx;
            if (a.arg[o] >= 0) k = snr_key(a.best[o], a.arg[o]);
        }
        keys[q] = k;
    }
    const bool full = x0 + 31 < a.w && y0 + P - 1 < a.h;
    const float inv_n = a.inv_sqrt[a.n];
    for (int g = a.g0; g < a.g1; ++g) {
        const StackGroup G = a.groups[g];
        uint16_t* offs = reinterpret_cast<uint16_t*>(win + G.rows_total * WP);
        if (!stage_group<NW, WP, BH>(a, G, g, tmap, x0, y0, bar, win, offs, block_next, err, phase)) return false;
        const bool interior = full && x0 + G.gdxmin >= 0 && x0 + 31 + G.gdxmax < a.w && y0 + G.gdymin >= 0 &&
                              y0 + P - 1 + G.gdymax < a.h;
        if (G.rows_fast) {
            if (interior) {
                for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                    motion_quad_rows_atom<P, WP, shape_row_spread(P, 1)>(a, G, s0, win, offs, tb, inv_n, keys);
            } else {
                for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                    motion_quad_rows_border_atom<P, WP, shape_row_spread(P, 1)>(a, G, s0, win, offs, tb, x, y0, keys);
            }
        } else if (interior) {
            for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                motion_quad_atom<P, WP, false>(a, G, s0, win, offs, tb, x, x0, y0, inv_n, keys);
        } else {
            for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                motion_quad_atom<P, WP, true>(a, G, s0, win, offs, tb, x, x0, y0, inv_n, keys);
        }
    }
    __syncthreads();
    for (int q = tid; q < 32 * P; q += 32 * NW) {
        const int xx = x0 + (q & 31), yy = y0 + (q >> 5);
        if (xx >= a.w || yy >= a.h) continue;
        const size_t o = static_cast<size_t>(yy) * a.w + xx;
        float b = -CUDART_INF_F;
        int ar = -1;
        if (keys[q] != 0ull) snr_unkey(keys[q], b, ar);
        if (a.last) {
            a.max_snr[o] = isfinite(b) ? b : 0.0f;
            a.best_v[o] = ar;
        } else {
            a.best[o] = b;
            a.arg[o] = ar;
        }
    }
    __syncthreads();  // the keys are reset by the next tile
    return true;
}

// ---- paired columns: each thread owns two adjacent columns of P rows, so a
// warp covers a 64-wide tile. Every add is a packed add.rn.f32x2 on the pair
// (two independent round-to-nearest float adds, bit-identical to two scalar
// adds), which halves the add instructions; a window offset that is even loads
// both columns with one 64-bit shared load, an odd one with two 32-bit loads.

template <int P, int WP>
__device__ __forceinline__ void load_pairs(float2 (&v)[P], const float* __restrict__ src, uint32_t odd) {
    if (!odd) {
#pragma unroll
        for (int p = 0; p < P; ++p) v[p] = *reinterpret_cast<const float2*>(src + p * WP);
    } else {
#pragma unroll
        for (int p = 0; p < P; ++p) v[p] = make_float2(src[p * WP], src[p * WP + 1]);
    }
}

template <int P>
__device__ __forceinline__ void add_pairs(float2 (&acc)[P], const float2 (&v)[P]) {
#pragma unroll
    for (int p = 0; p < P; ++p) acc[p] = __fadd2_rn(acc[p], v[p]);
}

// motion_quad for paired columns: x is the thread's first column
template <int P, int WP, bool BORDER>
__device__ __forceinline__ void motion_quad2(const StackArgs& a, const StackGroup& G, int s0,
                                             const float* __restrict__ win, const uint16_t* __restrict__ offs, int tb,
                                             int x, int x0, int y0, float inv_n, float (&best)[P][2],
                                             int (&arg)[P][2]) {
    constexpr int M = 4;
    constexpr int PW = (P + 3) / 4;
    float2 acc[M][P];
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int p = 0; p < P; ++p) acc[k][p] = make_float2(0.0f, 0.0f);
    int cfull[M] = {0, 0, 0, 0};
    uint32_t cpart[M][2][PW];
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int w = 0; w < PW; ++w) cpart[k][c][w] = 0;
    const uint16_t* op = offs + s0;
    uint2 qn = *reinterpret_cast<const uint2*>(op);
    const int n = a.n;
    for (int i = 0; i < n; ++i) {
        const uint2 q = qn;
        if (i + 1 < n) qn = *reinterpret_cast<const uint2*>(op + (i + 1) * G.nslots);
        const uint32_t o0 = q.x & 0xffffu, o1 = q.x >> 16, o2 = q.y & 0xffffu, o3 = q.y >> 16;
        float2 v[P];
        load_pairs<P, WP>(v, win + o0 + tb, o0 & 1u);
        add_pairs<P>(acc[0], v);
        if (o1 != o0) load_pairs<P, WP>(v, win + o1 + tb, o1 & 1u);
        add_pairs<P>(acc[1], v);
        if (o2 != o1) load_pairs<P, WP>(v, win + o2 + tb, o2 & 1u);
        add_pairs<P>(acc[2], v);
        if (o3 != o2) load_pairs<P, WP>(v, win + o3 + tb, o3 & 1u);
        add_pairs<P>(acc[3], v);
        if constexpr (BORDER) {
#pragma unroll
            for (int k = 0; k < M; ++k) {
                const short2 sh = a.slot_shift[static_cast<size_t>(G.slot0 + s0 + k) * n + i];
                const bool whole = x0 + sh.x >= 0 && x0 + 63 + sh.x < a.w && y0 + sh.y >= 0 && y0 + P - 1 + sh.y < a.h;
                if (whole) {
                    ++cfull[k];
                } else {
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const bool inx = static_cast<unsigned>(x + c + sh.x) < static_cast<unsigned>(a.w);
#pragma unroll
                        for (int p = 0; p < P; ++p)
                            if (inx && static_cast<unsigned>(y0 + p + sh.y) < static_cast<unsigned>(a.h))
                                cpart[k][c][p / 4] += 1u << (8 * (p % 4));
                    }
                }
            }
        }
    }
    const float2 inv2 = make_float2(inv_n, inv_n);
#pragma unroll
    for (int k = 0; k < M; ++k) {
        const int j = a.slot_motion[G.slot0 + s0 + k];
        if (j < 0) continue;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            float s[2];
            if constexpr (BORDER) {
                bool ok[2];
                float f[2];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int cc = cfull[k] + static_cast<int>((cpart[k][c][p / 4] >> (8 * (p % 4))) & 0xffu);
                    ok[c] = cc >= a.min_count;
                    f[c] = a.inv_sqrt[ok[c] ? cc : 0];
                }
                const float2 sn = __fmul2_rn(acc[k][p], make_float2(f[0], f[1]));
                s[0] = sn.x;
                s[1] = sn.y;
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (ok[c] && (s[c] > best[p][c] || (s[c] == best[p][c] && j < arg[p][c]))) {
                        best[p][c] = s[c];
                        arg[p][c] = j;
                    }
            } else {
                const float2 sn = __fmul2_rn(acc[k][p], inv2);
                s[0] = sn.x;
                s[1] = sn.y;
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    if (s[c] > best[p][c] || (s[c] == best[p][c] && j < arg[p][c])) {
                        best[p][c] = s[c];
                        arg[p][c] = j;
                    }
            }
        }
    }
}

// One 64 x P output tile of one pass with paired columns (as stack_tile).
template <int NW, int P, int WP, int BH>
__device__ bool stack_tile2(const StackArgs& a, const CUtensorMap* tmap, int x0, int y0, uint64_t* bar, float* win,
                            int* block_next, int* err, uint32_t& phase) {
    constexpr int M = 4;
    constexpr int TW = 64;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x = x0 + 2 * lane;
    const int tb = 2 * lane;

    float best[P][2];
    int arg[P][2];
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            best[p][c] = -CUDART_INF_F;
            arg[p][c] = -1;
        }
    const bool full = x0 + TW - 1 < a.w && y0 + P - 1 < a.h;
    const float inv_n = a.inv_sqrt[a.n];
    for (int g = a.g0; g < a.g1; ++g) {
        const StackGroup G = a.groups[g];
        uint16_t* offs = reinterpret_cast<uint16_t*>(win + G.rows_total * WP);
        if (!stage_group<NW, WP, BH>(a, G, g, tmap, x0, y0, bar, win, offs, block_next, err, phase)) return false;
        const bool interior = full && x0 + G.gdxmin >= 0 && x0 + TW - 1 + G.gdxmax < a.w && y0 + G.gdymin >= 0 &&
                              y0 + P - 1 + G.gdymax < a.h;
        if (interior) {
            for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                motion_quad2<P, WP, false>(a, G, s0, win, offs, tb, x, x0, y0, inv_n, best, arg);
        } else {
            for (int s0 = warp * M; s0 < G.nslots; s0 = next_block(block_next) * M)
                motion_quad2<P, WP, true>(a, G, s0, win, offs, tb, x, x0, y0, inv_n, best, arg);
        }
    }
    __syncthreads();
    float* mb = win;
    int* ma = reinterpret_cast<int*>(win + NW * TW * P);
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            mb[(warp * P + p) * TW + tb + c] = best[p][c];
            ma[(warp * P + p) * TW + tb + c] = arg[p][c];
        }
    __syncthreads();
    for (int q = tid; q < TW * P; q += 32 * NW) {
        const int p = q / TW, l = q % TW;
        const int xx = x0 + l, yy = y0 + p;
        if (xx >= a.w || yy >= a.h) continue;
        const size_t o = static_cast<size_t>(yy) * a.w + xx;
        float b = -CUDART_INF_F;
        int ar = -1;
        if (!a.first) {
            b = a.best[o];
            ar = a.arg[o];
        }
        for (int w = 0; w < NW; ++w) {
            const float s = mb[(w * P + p) * TW + l];
            const int j = ma[(w * P + p) * TW + l];
            if (j >= 0 && (s > b || (s == b && (ar < 0 || j < ar)))) {
                b = s;
                ar = j;
            }
        }
        if (a.last) {
            a.max_snr[o] = isfinite(b) ? b : 0.0f;
            a.best_v[o] = ar;
        } else {
            a.best[o] = b;
            a.arg[o] = ar;
        }
    }
    __syncthreads();
    return true;
}

// Persistent: one CTA per SM takes (pass, tile) work items from a queue until the
// batch is done, so passes of different shapes and sizes share one launch and
// the SMs stay busy to the end. TW: tile width, 32 (one column per thread) or
// 64 (paired columns).
template <int NW, int P, int WP, int BH, int TW, int MERGE>
__global__ void __launch_bounds__(32 * NW, 1)
    stack_batch_kernel(const StackArgs* __restrict__ passes, const CUtensorMap* __restrict__ maps, int npasses,
                       long long items, int* queue, int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // 128-byte aligned base (TMA destinations), the barrier in its first 8 bytes
    unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base);
    long long* next = reinterpret_cast<long long*>(base + 8);
    int* block_next = reinterpret_cast<int*>(base + 16);  // the current group's next 4-motion block
    // MERGE: the tile's shared maximum (32 x P keys) ahead of the windows
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(base + 128);
    float* win = reinterpret_cast<float*>(base + 128 + (MERGE ? 32 * P * 8 : 0));
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) *next = atomicAdd(reinterpret_cast<unsigned long long*>(queue), 1ull);
        __syncthreads();
        const long long item = *next;
        __syncthreads();
        if (item >= items) break;
        int p = 0;
        while (p + 1 < npasses && passes[p + 1].item0 <= item) ++p;
        const StackArgs& a = passes[p];
        const long long t = item - a.item0;
        const int tx = static_cast<int>(t % a.tiles_x), ty = a.ty0 + static_cast<int>(t / a.tiles_x);
        if constexpr (TW == 64) {
            if (!stack_tile2<NW, P, WP, BH>(a, maps + p, tx * 64, ty * P, bar, win, block_next, err, phase)) return;
        } else if constexpr (MERGE == 1) {
            if (!stack_tile_atom<NW, P, WP, BH>(a, maps + p, tx * 32, ty * P, bar, keys, win, block_next, err, phase))
                return;
        } else {
            if (!stack_tile<NW, P, WP, BH>(a, maps + p, tx * 32, ty * P, bar, win, block_next, err, phase)) return;
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw CudaError("cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

template <int NW, int P, int WP, int BH, int TW, int MERGE>
void launch_batch(const std::vector<BatchPass>& batch, unsigned char* d_desc, size_t desc_bytes, int* d_err,
                  int sms, cudaStream_t s) {
    const size_t np = batch.size();
    std::vector<unsigned char> host(batch_desc_bytes(static_cast<int>(np)), 0);
    if (host.size() > desc_bytes) throw std::runtime_error("stack batch: descriptor buffer too small");
    CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(host.data() + 128);
    StackArgs* args = reinterpret_cast<StackArgs*>(host.data() + 128 + 128 * np);
    long long items = 0;
    // the warps' maxima at the end of a tile, or (MERGE) the shared keys ahead of the windows
    const size_t keys_bytes = MERGE ? static_cast<size_t>(32) * P * 8 : 0;
    size_t smem = MERGE ? 256 + keys_bytes : 256 + static_cast<size_t>(NW) * TW * P * 8;
    for (size_t k = 0; k < np; ++k) {
        const BatchPass& bp = batch[k];
        const StackPlan& plan = *bp.plan;
        if (plan.cfg.ty != NW || plan.cfg.p != P || plan.cfg.tile_w != TW || plan.cfg.wp != WP || plan.cfg.merge != MERGE)
            throw std::runtime_error("stack batch: passes of different kernel shapes");
        const cuuint64_t dims[3] = {static_cast<cuuint64_t>(plan.w), static_cast<cuuint64_t>(plan.h),
                                    static_cast<cuuint64_t>(plan.n)};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(plan.pitch) * 4,
                                       static_cast<cuuint64_t>(plan.pitch) * plan.h * 4};
        const cuuint32_t box[3] = {WP, BH, 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        const CUresult r = encode_fn()(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(bp.frames), dims,
                                       strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            throw CudaError("cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")");
        StackArgs& a = args[k];
        a.w = plan.w;
        a.h = plan.h;
        a.n = plan.n;
        a.min_count = plan.min_count;
        a.g0 = bp.g0;
        a.g1 = bp.g1;
        a.first = bp.first;
        a.last = bp.last;
        a.tiles_x = (plan.w + TW - 1) / TW;
        a.tiles_y = (plan.h + P - 1) / P;
        a.ty0 = 0;
        if (bp.tile_rows > 0) {  // a band of tile rows (autotuning probes)
            a.ty0 = std::min(std::max(0, bp.tile_rows0), a.tiles_y - 1);
            a.tiles_y = std::min(bp.tile_rows, a.tiles_y - a.ty0);
        }
        a.item0 = items;
        items += static_cast<long long>(a.tiles_x) * a.tiles_y;
        const StackPlanDev& dev = *bp.dev;
        a.groups = dev.groups;
        a.wins = dev.wins;
        a.slot_motion = dev.slot_motion;
        a.slot_off = dev.slot_off;
        a.slot_off_base = dev.slot_off_base;
        a.slot_shift = dev.slot_shift;
        a.inv_sqrt = dev.inv_sqrt;
        a.best = bp.best;
        a.arg = bp.arg;
        a.max_snr = bp.max_snr;
        a.best_v = bp.best_v;
        a.err = d_err;
        a.extra_tx = static_cast<unsigned>(g_wait_extra.load());
        a.wait_limit = g_wait_extra.load() > 0 ? g_wait_cycles.load() : 4000000000LL;
        smem = std::max(smem, 256 + keys_bytes + static_cast<size_t>(plan.max_group_bytes));
        if (smem > static_cast<size_t>(plan.cfg.smem_bytes) + 256 + keys_bytes)
            throw std::runtime_error("stack plan exceeds shared memory");
    }
    if (items == 0) return;
    FTB_CHECK(cudaMemcpyAsync(d_desc, host.data(), host.size(), cudaMemcpyHostToDevice, s));
    auto kern = stack_batch_kernel<NW, P, WP, BH, TW, MERGE>;
    allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    const int ctas = static_cast<int>(std::min<long long>(items, sms));
    kern<<<ctas, 32 * NW, smem, s>>>(reinterpret_cast<const StackArgs*>(d_desc + 128 + 128 * np),
                                     reinterpret_cast<const CUtensorMap*>(d_desc + 128), static_cast<int>(np), items,
                                     reinterpret_cast<int*>(d_desc), d_err);
    FTB_CHECK(cudaGetLastError());
}

}  // namespace

size_t batch_desc_bytes(int npasses) {
    return 128 + 128 * static_cast<size_t>(npasses) + sizeof(StackArgs) * static_cast<size_t>(npasses);
}

void stack_launch_batch(const std::vector<BatchPass>& batch, unsigned char* d_desc, size_t desc_bytes, int* d_err,
                        int sms, cudaStream_t s) {
    if (batch.empty()) return;
    const StackConfig& c = batch[0].plan->cfg;
    if (c.bh != 4 || c.mblock != 4) throw std::runtime_error("stack: unsupported kernel configuration");
    if (c.tile_w == 64 && c.wp == 72 && c.ty == 12 && c.p == 8 && c.merge == 0)
        launch_batch<12, 8, 72, 4, 64, 0>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 12 && c.p == 16 && c.merge == 0)
        launch_batch<12, 16, 40, 4, 32, 0>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 16 && c.p == 8 && c.merge == 0)
        launch_batch<16, 8, 40, 4, 32, 0>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 16 && c.p == 4 && c.merge == 0)
        launch_batch<16, 4, 40, 4, 32, 0>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 16 && c.p == 16 && c.merge == 1)
        launch_batch<16, 16, 40, 4, 32, 1>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 14 && c.p == 16 && c.merge == 1)
        launch_batch<14, 16, 40, 4, 32, 1>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 16 && c.p == 12 && c.merge == 0)
        launch_batch<16, 12, 40, 4, 32, 0>(batch, d_desc, desc_bytes, d_err, sms, s);
    else if (c.tile_w == 32 && c.wp == 40 && c.ty == 16 && c.p == 20 && c.merge == 1)
        launch_batch<16, 20, 40, 4, 32, 1>(batch, d_desc, desc_bytes, d_err, sms, s);

    else
        throw std::runtime_error("stack: unsupported tile shape");
}

}  // namespace ftb
