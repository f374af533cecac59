// The "b200" stacking backend for FaintTrail's plugin interface.
//
// A SearchBackend (FaintTrail include/fainttrail/backend.hpp:107-117) whose
// run() forwards the pass to ft_b200_stack (include/ft_b200.h). Registered with
// register_backend("b200", ...) (backend.hpp:131-132, backend.cpp:27-35), it is
// selected by name -- SearchParams::backend = "b200", or ft_params.backend in
// the C API -- and then every real and null stacking pass of FaintTrail's
// search() runs on the B200 with bit-identical results.
//
// Build (against the FaintTrail headers, linking libft_b200.so):
//   g++ -std=c++17 -fPIC -shared -I<FaintTrail>/include -I<this repo>/include \
//       b200_backend.cpp -o libft_b200_adapter.so -L<dir of libft_b200.so> -lft_b200
// and load it into a process that has the FaintTrail library loaded; call
// ft_b200_register_backend() once.
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "fainttrail/backend.hpp"
#include "ft_b200.h"

namespace {

using namespace fainttrail;

class B200Backend final : public SearchBackend {
public:
    B200Backend() {
        if (ft_b200_open(-1, 0.0, &ctx_) != FT_B200_OK)
            throw std::runtime_error(std::string("b200 backend unavailable: ") + ft_b200_last_error(nullptr));
    }
    ~B200Backend() override { ft_b200_close(ctx_); }

    std::string name() const override { return "b200"; }

    std::string description() const override {
        char dev[128] = {0};
        int sms = 0;
        double mem = 0;
        ft_b200_device_info(ctx_, dev, sizeof dev, &sms, &mem);
        return std::string("B200 backend (sm_100a kernels): ") + dev + ", " + std::to_string(sms) + " SMs, " +
               std::to_string(static_cast<int>(mem / 1073741824.0)) + " GB";
    }

    StackResult run(const StackPass& pass, const ProgressFn& progress) override {
        validate_pass(pass);
        const auto& frames = *pass.frames;
        const int w = frames[0].width, h = frames[0].height, n = static_cast<int>(frames.size());
        const int m = pass_motions(pass);
        // the frames as one host block, and the shifts as a motion-major table
        // (exactly pass_shift, backend.hpp:87-97, for straight and explicit tracks)
        std::vector<float> block(static_cast<size_t>(w) * h * n);
        for (int i = 0; i < n; ++i)
            std::memcpy(block.data() + static_cast<size_t>(i) * w * h, frames[static_cast<size_t>(i)].data.data(),
                        sizeof(float) * static_cast<size_t>(w) * h);
        std::vector<int> dx(static_cast<size_t>(m) * n), dy(dx.size());
        for (int j = 0; j < m; ++j)
            for (int i = 0; i < n; ++i)
                pass_shift(pass, j, i, dx[static_cast<size_t>(j) * n + i], dy[static_cast<size_t>(j) * n + i]);
        StackResult out;
        out.max_snr = Image(w, h);
        out.best_v.assign(static_cast<size_t>(w) * h, -1);
        struct Cb {
            const ProgressFn* fn;
        } cb{&progress};
        auto tramp = [](double f, const char* stage, void* user) -> int {
            const ProgressFn& fn = *static_cast<Cb*>(user)->fn;
            return fn(f, stage ? stage : "stack") ? 1 : 0;
        };
        const int rc = ft_b200_stack(ctx_, block.data(), w, h, n, dx.data(), dy.data(), m, pass.min_count,
                                     out.max_snr.data.data(), out.best_v.data(), progress ? +tramp : nullptr, &cb);
        if (rc == FT_B200_CANCELLED) throw Cancelled();
        if (rc != FT_B200_OK) throw std::runtime_error(std::string("b200 backend: ") + ft_b200_last_error(ctx_));
        char names[512] = {0};
        double secs[16] = {0};
        const int k = ft_b200_timings(ctx_, names, sizeof names, secs, 16);
        std::string all(names);
        size_t start = 0;
        for (int t = 0; t < k && t < 16; ++t) {
            const size_t end = all.find(';', start);
            out.timings.push_back({all.substr(start, end == std::string::npos ? std::string::npos : end - start),
                                   secs[t]});
            if (end == std::string::npos) break;
            start = end + 1;
        }
        if (progress) progress(1.0, "stack");
        return out;
    }

private:
    ft_b200_ctx* ctx_ = nullptr;
};

}  // namespace

extern "C" int ft_b200_register_backend(void) {
    try {
        register_backend("b200", [] { return std::unique_ptr<SearchBackend>(new B200Backend()); });
        return 0;
    } catch (...) {
        return 1;
    }
}
