// beamformer_cuda -- command-line beamformer over the B200 backend.
//
// A drop-in for the reference's tools/beamformer_cuda.cpp: the same options,
// input and output files, stdout report and metrics CSV row, so scripts that
// drive the reference tool (its validation runner included) run unchanged.
// Additions: --kernel tensor selects the split-precision tensor-core path,
// --kernel covariance the opt-in covariance form and --kernel checked the
// covariance form with split-precision recomputation wherever its error
// estimate is too high (all take canonical weights, like direct).
//
//   beamformer_cuda --input V --weights W --output O [--n-time N] [--n-ant N]
//       [--n-beams N] [--kernel direct|tiled|tensor|covariance|checked] [--integration-spectra S]
//       [--output-format float32|int8 --quantization-params P
//        --quantization-metadata M] [--shard-id 0|1] [--metrics CSV]
//
// Exit status 0 on success, 1 with "beamformer_cuda: <message>" on stderr.
#include "beamformer/config.hpp"
#include "beamformer/cuda_beamformer.hpp"
#include "beamformer/io.hpp"

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstdlib>
#include <exception>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <optional>
#include <stdexcept>
#include <string>
#include <system_error>
#include <vector>

namespace {

namespace bf = beamformer;
using Clock = std::chrono::steady_clock;

struct Args {
    std::filesystem::path input, weights, output;
    std::optional<std::filesystem::path> metrics, params, metadata;
    std::size_t n_time = 15360, n_ant = 64, n_beams = 5, shard_id = 0;
    std::optional<std::size_t> spectra;
    bool int8 = false;
    bf::CudaBeamformerKernel kernel = bf::CudaBeamformerKernel::Direct;
};

void usage(const char* prog) {
    std::cout << "Usage: " << prog << " --input FILE --weights FILE --output FILE [options]\n\n"
              << "  --n-time N              default: 15360\n"
              << "  --n-ant N               32 or 64; default: 64\n"
              << "  --n-beams N             1 to 128; default: 5\n"
              << "  --kernel NAME           direct, tiled, tensor, covariance or checked; default: direct\n"
              << "  --integration-spectra N GPU integration: 10 or 320\n"
              << "  --output-format NAME    float32 or int8; default: float32\n"
              << "  --quantization-params F int8 parameter output; required for int8\n"
              << "  --quantization-metadata F int8 metadata output; required for int8\n"
              << "  --shard-id N            0 or 1; default: 0\n"
              << "  --metrics FILE          append timing row to CSV\n";
}

std::size_t to_size(const std::string& text, const std::string& option) {
    std::size_t used = 0;
    const unsigned long long v = std::stoull(text, &used);
    if (used != text.size()) throw std::invalid_argument("invalid integer for " + option);
    return static_cast<std::size_t>(v);
}

Args parse(int argc, char** argv) {
    Args a;
    auto value = [&](int& i) -> std::string {
        if (i + 1 >= argc) throw std::invalid_argument(std::string("missing value after ") + argv[i]);
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        const std::string opt = argv[i];
        if (opt == "--help") {
            usage(argv[0]);
            std::exit(0);
        } else if (opt == "--input") {
            a.input = value(i);
        } else if (opt == "--weights") {
            a.weights = value(i);
        } else if (opt == "--output") {
            a.output = value(i);
        } else if (opt == "--metrics") {
            a.metrics = value(i);
        } else if (opt == "--n-time") {
            a.n_time = to_size(value(i), opt);
        } else if (opt == "--n-ant") {
            a.n_ant = to_size(value(i), opt);
        } else if (opt == "--n-beams") {
            a.n_beams = to_size(value(i), opt);
        } else if (opt == "--kernel") {
            const std::string k = value(i);
            if (k == "direct") a.kernel = bf::CudaBeamformerKernel::Direct;
            else if (k == "tiled") a.kernel = bf::CudaBeamformerKernel::Tiled;
            else if (k == "tensor") a.kernel = bf::CudaBeamformerKernel::TensorSplit;
            else if (k == "covariance") a.kernel = bf::CudaBeamformerKernel::TensorCovariance;
            else if (k == "checked") a.kernel = bf::CudaBeamformerKernel::TensorChecked;
            else throw std::invalid_argument("kernel must be direct, tiled, tensor, covariance or checked");
        } else if (opt == "--integration-spectra") {
            a.spectra = to_size(value(i), opt);
        } else if (opt == "--output-format") {
            const std::string f = value(i);
            if (f == "float32") a.int8 = false;
            else if (f == "int8") a.int8 = true;
            else throw std::invalid_argument("output format must be float32 or int8");
        } else if (opt == "--quantization-params") {
            a.params = value(i);
        } else if (opt == "--quantization-metadata") {
            a.metadata = value(i);
        } else if (opt == "--shard-id") {
            a.shard_id = to_size(value(i), opt);
        } else {
            throw std::invalid_argument("unknown option: " + opt);
        }
    }
    if (a.input.empty() || a.weights.empty() || a.output.empty()) {
        throw std::invalid_argument("--input, --weights, and --output are required");
    }
    if (a.int8 && (!a.spectra || !a.params || !a.metadata)) {
        throw std::invalid_argument(
            "int8 output requires --integration-spectra, --quantization-params, and --quantization-metadata");
    }
    if (a.shard_id >= bf::frequency_shard_count) throw std::invalid_argument("--shard-id must be 0 or 1");
    return a;
}

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

const char* kernel_name(bf::CudaBeamformerKernel k) {
    switch (k) {
        case bf::CudaBeamformerKernel::Direct: return "direct";
        case bf::CudaBeamformerKernel::Tiled: return "tiled";
        case bf::CudaBeamformerKernel::TensorCovariance: return "covariance";
        case bf::CudaBeamformerKernel::TensorChecked: return "checked";
        default: return "tensor";
    }
}

// beam with the largest sum over all (time, frequency) outputs
std::size_t brightest_beam(const bf::Intensities& v, std::size_t n_beams) {
    std::vector<double> sum(n_beams, 0.0);
    for (std::size_t i = 0; i < v.size(); ++i) sum[i % n_beams] += v[i];
    return static_cast<std::size_t>(std::distance(sum.begin(), std::max_element(sum.begin(), sum.end())));
}

struct Report {
    double load = 0, unpack = 0, setup = 0, h2d = 0, compute = 0, d2h = 0, write = 0, total = 0;
};

void append_csv(const std::filesystem::path& path, const bf::Dimensions& d, const Report& r, double out_rate,
                double gmac_rate) {
    std::error_code ec;
    const bool exists = std::filesystem::exists(path, ec);
    if (ec) throw std::runtime_error("cannot inspect metrics file: " + path.string());
    const std::uintmax_t size = exists ? std::filesystem::file_size(path, ec) : 0;
    if (ec) throw std::runtime_error("cannot inspect metrics file: " + path.string());
    std::ofstream out(path, std::ios::app);
    if (!out) throw std::runtime_error("cannot open metrics file: " + path.string());
    if (!exists || size == 0) {
        out << "backend,n_time,n_freq,n_ant,n_beams,load_ms,unpack_ms,setup_ms,host_to_device_ms,compute_ms,"
               "device_to_host_ms,write_ms,total_ms,output_elements_per_second,complex_gmac_per_second\n";
    }
    out << std::fixed << std::setprecision(6) << "cuda," << d.n_time << ',' << d.n_freq << ',' << d.n_ant << ','
        << d.n_beams << ',' << r.load << ',' << r.unpack << ',' << r.setup << ',' << r.h2d << ',' << r.compute
        << ',' << r.d2h << ',' << r.write << ',' << r.total << ',' << out_rate << ',' << gmac_rate << '\n';
    if (!out) throw std::runtime_error("failed to write metrics file: " + path.string());
}

int run(const Args& a) {
    const bf::Dimensions dims{a.n_time, bf::default_frequency_channels, a.n_ant, a.n_beams};
    bf::validate_dimensions(dims);
    const auto t0 = Clock::now();
    const bf::PackedVoltage packed = bf::read_packed_voltage(a.input, dims);
    const bf::Weights weights = a.kernel == bf::CudaBeamformerKernel::Tiled ? bf::read_tiled_weights(a.weights, dims)
                                                                            : bf::read_weights(a.weights, dims);
    const auto t_load = Clock::now();
    bf::CudaBeamformerTimings ct;
    std::optional<bf::TemporalIntegrationConfig> integ;
    if (a.spectra) integ = bf::TemporalIntegrationConfig{*a.spectra};
    const bf::Dimensions out_dims =
        integ ? bf::Dimensions{bf::integrated_time_count(dims.n_time, *integ), dims.n_freq, dims.n_ant, dims.n_beams}
              : dims;
    std::size_t out_bytes = 0, out_elements = 0;
    std::optional<std::size_t> peak;
    Clock::time_point t_compute;
    if (a.int8) {
        const auto q = bf::cuda_beamform_packed_quantized_integrated_intensity(packed, weights, dims, *integ, &ct,
                                                                               a.kernel);
        t_compute = Clock::now();
        bf::write_quantized_intensities(a.output, q.codes, out_dims);
        bf::write_quantization_parameters(*a.params, q.parameters, out_dims);
        bf::write_quantized_output_metadata(
            *a.metadata, bf::QuantizedOutputMetadata{out_dims, dims.n_time, *integ,
                                                     bf::default_shard_descriptors()[a.shard_id],
                                                     a.params->filename().string()});
        out_elements = q.codes.size();
        out_bytes = q.codes.size() + q.parameters.size() * sizeof(bf::Int8QuantizationParameters);
    } else {
        const bf::Intensities v = integ ? bf::cuda_beamform_packed_integrated_intensity(packed, weights, dims, *integ,
                                                                                        &ct, a.kernel)
                                        : bf::cuda_beamform_packed_intensity(packed, weights, dims, &ct, a.kernel);
        t_compute = Clock::now();
        bf::write_intensities(a.output, v, out_dims);
        out_elements = v.size();
        out_bytes = v.size() * sizeof(float);
        peak = brightest_beam(v, out_dims.n_beams);
    }
    const auto t_write = Clock::now();

    Report r;
    r.load = ms_between(t0, t_load);
    r.unpack = 0.0;  // the packed bytes are decoded inside the kernels
    r.setup = ct.setup_ms;
    r.h2d = ct.host_to_device_ms;
    r.compute = ct.kernel_ms + ct.temporal_integration_ms + ct.quantization_ms;
    r.d2h = ct.device_to_host_ms;
    r.write = ms_between(t_compute, t_write);
    r.total = ms_between(t0, t_write);
    const double secs = r.compute / 1000.0;
    const double outs = static_cast<double>(out_elements);
    const double cmacs = static_cast<double>(dims.n_time * dims.n_freq * dims.n_beams) * static_cast<double>(dims.n_ant);
    const double out_rate = secs > 0.0 ? outs / secs : 0.0;
    const double gmac_rate = secs > 0.0 ? cmacs / secs / 1.0e9 : 0.0;
    const double call_ms = ms_between(t_load, t_compute);
    const double pipe_ms = r.h2d + r.compute + r.d2h;
    const double pipe_rate = pipe_ms > 0.0 ? outs / (pipe_ms / 1000.0) : 0.0;
    if (a.metrics) append_csv(*a.metrics, dims, r, out_rate, gmac_rate);

    std::cout << std::fixed << std::setprecision(3) << "CUDA beamforming complete: kernel=" << kernel_name(a.kernel)
              << " input_layout=[T=" << dims.n_time << "][F=" << dims.n_freq << "][B=" << dims.n_beams << "]"
              << " output_layout=[T=" << out_dims.n_time << "][F=" << out_dims.n_freq << "][B=" << out_dims.n_beams
              << "]\n"
              << "load_ms=" << r.load << " unpack_ms=" << r.unpack << " setup_ms=" << r.setup
              << " host_to_device_ms=" << r.h2d << " kernel_ms=" << r.compute << " beamformer_ms=" << ct.kernel_ms
              << " temporal_integration_ms=" << ct.temporal_integration_ms
              << " quantization_ms=" << ct.quantization_ms << " device_to_host_ms=" << r.d2h
              << " cuda_call_ms=" << call_ms << " write_ms=" << r.write << " total_ms=" << r.total << "\n"
              << "kernel_output_elements_per_second=" << out_rate
              << " pipeline_output_elements_per_second=" << pipe_rate << " complex_GMAC_per_second=" << gmac_rate;
    if (peak) std::cout << " peak_integrated_beam=" << *peak;
    std::cout << "\nWrote " << out_bytes << " bytes of output data to " << a.output << "\n";
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(parse(argc, argv));
    } catch (const std::exception& e) {
        std::cerr << "beamformer_cuda: " << e.what() << "\n";
        return 1;
    }
}
