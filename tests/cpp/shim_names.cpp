// Builds (and is never run by the tests) the shim's sampler variants that carry the reference's
// other class names: SamplerGpuSectionedShared and SamplerRejectionGiveUp. Run with no
// arguments it does nothing; with one argument it builds a 4096-item table and draws from both.
#include <cstdio>
#include <vector>

#include "wrs.hpp"

int main(int argc, char** argv) {
    (void)argv;
    if (argc < 2) return 0;
    try {
        std::vector<float> w(4096);
        for (size_t i = 0; i < w.size(); ++i) w[i] = 1.0f + (float)(i % 7);
        wrs::AliasTableSplitGpu a(w);
        if (!a.fullBuild()) return 1;
        wrs::SamplerGpuSectionedShared s(a);
        wrs::RejectionSamplingGpu r(w);
        if (!r.fullBuild()) return 1;
        wrs::SamplerRejectionGiveUp g(r);
        std::printf("%s %.3f %s %.3f\n", s.name().c_str(), s.benchmarkSampling(1 << 20), g.name().c_str(),
                    g.benchmarkSampling(1 << 20));
    } catch (const wrs::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
