// run_tracker_stream -- command-line beam tracker over the B200 backend.
//
// A drop-in for the reference's tools/run_tracker_stream.cpp, the program its
// astronomical validation runner drives: the same options, raw packed
// voltage in ([T][F][A] bytes), per-spectrum float32 intensity out
// ([T][F][1]), the same messages and exit codes.  Every CUDA engine name of
// the reference (cuda_fws, the default, cuda_twopass, cuda_fused, cuda_warp,
// cuda_v3*, cuda_v4*, cuda_v5*) runs the B200 streaming tracker; the CPU
// engine names (cpu_naive, cpu_v1, cpu_v2) belong to the reference's CPU
// library and are refused here with the reference's "unknown engine" error.
#include "beamformer/beam_tracker.hpp"
#include "beamformer/cuda_beam_tracker_v5.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/geometry.hpp"

#include <cstddef>
#include <exception>
#include <fstream>
#include <iostream>
#include <set>
#include <string>
#include <vector>

namespace {

namespace bf = beamformer;

void usage(const char* prog) {
    std::cout << "Usage: " << prog << " [options]\n"
              << "  --engine ENGINE       cuda_fws (default), cuda_twopass, cuda_fused, cuda_warp, cuda_v3, cuda_v4,\n"
              << "                        cuda_v5 and their variants: all run the B200 streaming tracker\n"
              << "  --n-time N            number of time samples\n"
              << "  --n-freq N            number of frequency channels (default 336)\n"
              << "  --n-ant N             number of antenna elements (32 or 64)\n"
              << "  --spectra N           integration spectra per window (default 320)\n"
              << "  --source-l0 L0        steering start l0\n"
              << "  --source-m0 M0        steering start m0\n"
              << "  --source-dl DL        steering rate dl/sample\n"
              << "  --source-dm DM        steering rate dm/sample\n"
              << "  --input FILE          input packed voltage binary file\n"
              << "  --output FILE         output float32 intensity binary file\n";
}

const std::set<std::string>& cuda_engines() {
    static const std::set<std::string> names = {
        "cuda_twopass", "cuda_fused", "cuda_warp", "cuda_fws", "cuda_v3", "cuda_v3_stream", "cuda_v3_direct",
        "cuda_v4", "cuda_v4_stream", "cuda_v4_direct", "cuda_v4_u4", "cuda_v4_u8", "cuda_v4_half2",
        "cuda_v5", "cuda_v5_u8", "cuda_v5_u4"};
    return names;
}

}  // namespace

int main(int argc, char** argv) {
    std::string engine = "cuda_fws";
    std::size_t n_time = 15360, n_freq = bf::default_frequency_channels, n_ant = 64, spectra = 320;
    float l0 = 0.0F, m0 = 0.0F, dl = 0.0F, dm = 0.0F;
    std::string input, output;
    try {
        // options the reference accepts, with its rule that an option missing
        // its value (or an unknown word) is skipped
        for (int i = 1; i < argc; ++i) {
            const std::string arg = argv[i];
            const bool has = i + 1 < argc;
            if (arg == "--engine" && has) engine = argv[++i];
            else if (arg == "--n-time" && has) n_time = std::stoull(argv[++i]);
            else if (arg == "--n-freq" && has) n_freq = std::stoull(argv[++i]);
            else if (arg == "--n-ant" && has) n_ant = std::stoull(argv[++i]);
            else if (arg == "--spectra" && has) spectra = std::stoull(argv[++i]);
            else if (arg == "--source-l0" && has) l0 = std::stof(argv[++i]);
            else if (arg == "--source-m0" && has) m0 = std::stof(argv[++i]);
            else if (arg == "--source-dl" && has) dl = std::stof(argv[++i]);
            else if (arg == "--source-dm" && has) dm = std::stof(argv[++i]);
            else if (arg == "--input" && has) input = argv[++i];
            else if (arg == "--output" && has) output = argv[++i];
            else if (arg == "--help" || arg == "-h") {
                usage(argv[0]);
                return 0;
            }
        }
        if (input.empty() || output.empty()) {
            std::cerr << "Error: --input and --output are required.\n";
            usage(argv[0]);
            return 1;
        }
        const bf::Dimensions dims{n_time, n_freq, n_ant, bf::tracker_beam_count};
        bf::TrackerConfig cfg;
        cfg.trajectory.direction_start = bf::direction_from_lm(l0, m0);
        cfg.trajectory.direction_rate_per_sample = {dl, dm};
        cfg.integration_spectra = spectra;

        std::ifstream in(input, std::ios::binary | std::ios::ate);
        if (!in) {
            std::cerr << "Error: Cannot open input file: " << input << "\n";
            return 1;
        }
        const std::size_t bytes = static_cast<std::size_t>(in.tellg());
        const std::size_t want = n_time * n_freq * n_ant;
        if (bytes != want) {
            std::cerr << "Error: Input file size (" << bytes << ") does not match expected (" << want << ")\n";
            return 1;
        }
        in.seekg(0);
        bf::PackedVoltage packed(want);
        in.read(reinterpret_cast<char*>(packed.data()), static_cast<std::streamsize>(want));
        if (!in) {
            std::cerr << "Error: Cannot read input file: " << input << "\n";
            return 1;
        }

        bf::Intensities intensity(n_time * n_freq * dims.n_beams, 0.0F);
        if (cuda_engines().count(engine) == 0) {
            std::cerr << "Error: Unknown engine or CUDA unavailable: " << engine << "\n";
            return 1;
        }
        bf::cuda_beam_tracker_v5_into(packed, dims, cfg, intensity);

        std::ofstream out(output, std::ios::binary);
        if (!out) {
            std::cerr << "Error: Cannot open output file: " << output << "\n";
            return 1;
        }
        out.write(reinterpret_cast<const char*>(intensity.data()),
                  static_cast<std::streamsize>(intensity.size() * sizeof(float)));
        out.close();
        std::cout << "Successfully ran " << engine << " on " << input << " -> wrote " << output << " ("
                  << intensity.size() * sizeof(float) << " bytes)\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 1;
    }
}
