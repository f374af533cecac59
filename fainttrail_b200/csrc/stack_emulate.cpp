// Host emulation of the stacking kernel (stack.cu) over its plan: the same
// output tiles, motion groups, per-frame windows (zero outside the frame, as
// the TMA copies fill them), 16-bit window offsets, clamped shifts for the
// coverage counts, float adds in ascending frame order, the 1/sqrt(c) scale and
// the maximum rule (larger S/N, or equal S/N and lower motion index), walked on
// the CPU; groups of blocks that share their column read the row descriptors
// the kernel reads. It lets the planner be checked against the stacking contract on a
// machine without a GPU, as the reference checks its CUDA algorithm with
// emulate_cuda_pass (cuda_plan.cpp:74-117).
#include <cmath>
#include <limits>
#include <stdexcept>
#include <vector>

#include "ft_internal.h"

namespace ftb {

void emulate_stack_pass(const StackPlan& P, const float* frames, float* max_snr, int* best_v) {
    const int w = P.w, h = P.h, n = P.n;
    const int TW = P.cfg.tile_w, TH = P.cfg.tile_h(), WP = P.cfg.wp;
    const int tiles_x = (w + TW - 1) / TW, tiles_y = (h + TH - 1) / TH;
    std::vector<float> win(static_cast<size_t>(P.max_rows) * WP);
    std::vector<float> best(static_cast<size_t>(TW) * TH);
    std::vector<int> arg(best.size());
    for (int ty = 0; ty < tiles_y; ++ty)
        for (int tx = 0; tx < tiles_x; ++tx) {
            const int x0 = tx * TW, y0 = ty * TH;
            std::fill(best.begin(), best.end(), -std::numeric_limits<float>::infinity());
            std::fill(arg.begin(), arg.end(), -1);
            for (size_t g = 0; g < P.groups.size(); ++g) {
                const StackGroup& G = P.groups[g];
                // the group's windows: frame i's rows [y0 + dy0, + rows) and columns
                // [x0 + dx0, + WP), zero outside the frame
                for (int i = 0; i < n; ++i) {
                    const StackWin& wv = P.wins[static_cast<size_t>(G.win0 + i)];
                    for (int r = 0; r < wv.rows; ++r) {
                        const int fy = y0 + wv.dy0 + r;
                        for (int c = 0; c < WP; ++c) {
                            const int fx = x0 + wv.dx0 + c;
                            const bool in = fx >= 0 && fx < w && fy >= 0 && fy < h;
                            win[static_cast<size_t>(wv.row0 + r) * WP + c] =
                                in ? frames[(static_cast<size_t>(i) * h + fy) * w + fx] : 0.0f;
                        }
                    }
                }
                // a tile inside the frame whose group shifts keep every window inside
                // it: every frame covers every pixel, c = n (the kernel's interior path)
                const bool interior = x0 + TW - 1 < w && y0 + TH - 1 < h && x0 + G.gdxmin >= 0 &&
                                      x0 + TW - 1 + G.gdxmax < w && y0 + G.gdymin >= 0 &&
                                      y0 + TH - 1 + G.gdymax < h;
                const uint16_t* offs = P.slot_off.data() + P.slot_off_base[g];
                // window offset of slot s in frame i: from the group's row
                // descriptors ([frame][block] words: lowest row's offset, each
                // slot's row above it) or its 16-bit slot table
                auto slot_offset = [&](int s, int i) -> size_t {
                    if (!G.rows_fast) return offs[static_cast<size_t>(i) * G.nslots + s];
                    const size_t e = 2 * (static_cast<size_t>(i) * (G.nslots / kMotionBlock) + s / kMotionBlock);
                    const uint32_t d = offs[e] | (static_cast<uint32_t>(offs[e + 1]) << 16);
                    return (d & 0xffffu) + ((d >> (16 + 2 * (s % kMotionBlock))) & 3u) * static_cast<size_t>(WP);
                };
                for (int s = 0; s < G.nslots; ++s) {
                    const int j = P.slot_motion[static_cast<size_t>(G.slot0 + s)];
                    if (j < 0) continue;  // a pad slot
                    const short2* sh = P.slot_shift.data() + static_cast<size_t>(G.slot0 + s) * n;
                    for (int yl = 0; yl < TH; ++yl)
                        for (int xl = 0; xl < TW; ++xl) {
                            float acc = 0.0f;
                            int c = 0;
                            for (int i = 0; i < n; ++i) {
                                const size_t o = slot_offset(s, i);
                                acc = acc + win[o + static_cast<size_t>(yl) * WP + xl];
                                const int cx = x0 + xl + sh[i].x, cy = y0 + yl + sh[i].y;
                                if (cx >= 0 && cx < w && cy >= 0 && cy < h) ++c;
                            }
                            if (interior) {
                                c = n;  // no count and no min_count test there
                            } else if (c < P.min_count) {
                                continue;
                            }
                            const float snr = acc * P.inv_sqrt[static_cast<size_t>(c)];
                            const size_t q = static_cast<size_t>(yl) * TW + xl;
                            if (snr > best[q] || (snr == best[q] && j < arg[q])) {
                                best[q] = snr;
                                arg[q] = j;
                            }
                        }
                }
            }
            for (int yl = 0; yl < TH; ++yl)
                for (int xl = 0; xl < TW; ++xl) {
                    const int xx = x0 + xl, yy = y0 + yl;
                    if (xx >= w || yy >= h) continue;
                    const size_t q = static_cast<size_t>(yl) * TW + xl, o = static_cast<size_t>(yy) * w + xx;
                    max_snr[o] = std::isfinite(best[q]) ? best[q] : 0.0f;
                    best_v[o] = arg[q];
                }
        }
}

}  // namespace ftb
