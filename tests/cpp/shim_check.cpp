// Exercises include/wrs.hpp, the C++ shim of the reference's object surface, end to end:
// builds the alias table and the rejection structure of the weights in a float32 file, draws
// plain, counted, sectioned and rejection samples, and writes them next to the output prefix
// for the test to compare with the oracle. Prints one JSON line.
//
//   shim_check <weights.f32> <out_prefix> <num_samples> <seed>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "wrs.hpp"

template <class T>
static void write_file(const std::string& path, const std::vector<T>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s weights.f32 out_prefix num_samples seed\n", argv[0]);
        return 2;
    }
    std::ifstream f(argv[1], std::ios::binary | std::ios::ate);
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<float> w((size_t)bytes / sizeof(float));
    f.read(reinterpret_cast<char*>(w.data()), bytes);
    const std::string out = argv[2];
    const uint64_t m = std::strtoull(argv[3], nullptr, 10);
    const uint64_t seed = std::strtoull(argv[4], nullptr, 10);
    try {
        wrs::AliasTableSplitGpu alias(w);
        if (!alias.fullBuild()) return 1;
        const std::vector<wrs_alias_row> rows = alias.hostTable();
        write_file(out + "_rows.bin", rows);

        wrs::SamplerGpuBasic basic(alias, seed);
        wrs::DeviceArray<uint32_t> d(m);
        basic.sample(m, d.get());  // counter 0
        write_file(out + "_plain.bin", d.to_host());
        write_file(out + "_hist.bin", basic.getSamplingDistribution(m));  // counter m

        wrs::SamplerGpuSectioned sect(alias, 4096, seed);
        sect.sample(m, d.get());
        write_file(out + "_sect.bin", d.to_host());

        wrs::RejectionSamplingGpu rej(w);
        if (!rej.fullBuild()) return 1;
        wrs::SamplerRejection rs(rej, seed);
        rs.sample(m, d.get());
        write_file(out + "_rej.bin", d.to_host());

        // the same weights cut into three tables, built as a batch and sampled 1000 times each
        const int64_t n = (int64_t)w.size();
        wrs::BatchedAliasTablesGpu batch(w, {0, n / 3, n / 2, n});
        if (!batch.fullBuild()) return 1;
        write_file(out + "_batch_rows.bin", batch.hostTable());
        wrs::SamplerBatched bs(batch, seed);
        write_file(out + "_batch_samples.bin", bs.sample({1000, 1000, 1000}));

        const double gs = wrs::SamplerGpuBasic(alias, seed).benchmarkSampling(m);
        std::printf("{\"alias\": \"%s\", \"W\": %.17g, \"rejection\": \"%s\", \"slots\": %llu, \"sampler\": \"%s\", "
                    "\"gsamples_per_s\": %.3f}\n",
                    alias.name().c_str(), alias.W, rej.name().c_str(), (unsigned long long)rej.slots,
                    basic.name().c_str(), gs);
    } catch (const wrs::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
