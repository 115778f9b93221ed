// test_io.cpp -- the on-disk formats of include/beamformer/io.hpp (CPU only).
//
//   test_io write SRC OUT   write every format into OUT from the raw arrays in
//                           SRC (voltage.raw, weights.raw, tiled.raw,
//                           intensity.raw, codes.raw, params.raw, loss.raw and
//                           dims.txt: T F A B S shard_id ts_start ts_step loss_id)
//   test_io read SRC DIR    read every format from DIR and compare with SRC
//   test_io errors DIR      error behaviour (types and the file-size check)
//
// tests/test_io_formats.py drives it against files written by the reference's
// own src/io.cpp: byte-identical output, and each side reads the other's.
#include "beamformer/io.hpp"

#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

namespace bf = beamformer;

namespace {

struct Case {
    std::size_t T, F, A, B, S, shard_id;
    std::uint64_t ts_start, ts_step, loss_id;
};

Case load_case(const std::string& src) {
    std::ifstream in(src + "/dims.txt");
    Case c{};
    if (!(in >> c.T >> c.F >> c.A >> c.B >> c.S >> c.shard_id >> c.ts_start >> c.ts_step >> c.loss_id)) {
        throw std::runtime_error("bad dims.txt");
    }
    return c;
}

template <typename T>
std::vector<T> raw(const std::string& path, std::size_t count) {
    std::ifstream in(path, std::ios::binary);
    std::vector<T> v(count);
    in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(count * sizeof(T)));
    if (!in) throw std::runtime_error("cannot read " + path);
    return v;
}

struct Data {
    bf::Dimensions d, wd;
    bf::PackedVoltage volt;
    bf::Weights w;
    bf::TiledWeights tw;
    bf::Intensities inten;
    bf::QuantizedIntensities codes;
    std::vector<bf::Int8QuantizationParameters> params;
    bf::LossMask loss;
    bf::ShardDescriptor shard;
    Case c;
};

Data load(const std::string& src) {
    Data x;
    x.c = load_case(src);
    const Case& c = x.c;
    x.d = bf::Dimensions{c.T, c.F, c.A, c.B};
    x.wd = bf::Dimensions{bf::integrated_time_count(c.T, bf::TemporalIntegrationConfig{c.S}), c.F, c.A, c.B};
    x.volt = raw<std::uint8_t>(src + "/voltage.raw", c.T * c.F * c.A);
    x.w = raw<bf::ComplexFloat>(src + "/weights.raw", c.B * c.F * c.A);
    x.tw = raw<bf::ComplexFloat>(src + "/tiled.raw", bf::tiled_weight_count(x.d));
    x.inten = raw<float>(src + "/intensity.raw", c.T * c.F * c.B);
    x.codes = raw<std::int8_t>(src + "/codes.raw", x.wd.n_time * c.F * c.B);
    x.params = raw<bf::Int8QuantizationParameters>(src + "/params.raw", bf::quantization_parameter_count(x.wd));
    x.loss = raw<std::uint8_t>(src + "/loss.raw", c.T * c.F);
    x.shard = bf::default_shard_descriptors()[c.shard_id];
    x.shard.timestamp_start = c.ts_start;
    x.shard.timestamp_step = c.ts_step;
    x.shard.loss_mask_id = c.loss_id;
    return x;
}

void write_all(const std::string& src, const std::string& out) {
    const Data x = load(src);
    bf::write_packed_voltage(out + "/voltage.bin", x.volt, x.d);
    bf::write_weights(out + "/weights.bin", x.w, x.d);
    bf::write_tiled_weights(out + "/tiled.bin", x.tw, x.d);
    bf::write_intensities(out + "/intensity.bin", x.inten, x.d);
    bf::write_quantized_intensities(out + "/codes.bin", x.codes, x.wd);
    bf::write_quantization_parameters(out + "/params.bin", x.params, x.wd);
    bf::write_quantized_output_metadata(
        out + "/int8_meta.txt",
        bf::QuantizedOutputMetadata{x.wd, x.c.T, bf::TemporalIntegrationConfig{x.c.S}, x.shard, "params.bin"});
    bf::write_packed_shard(out + "/shard_payload.bin", out + "/shard_meta.txt", out + "/shard_loss.bin",
                           bf::PackedShard{x.shard, x.volt, x.loss}, x.d);
    std::cout << "WRITE OK\n";
}

template <typename T>
void same(const std::vector<T>& a, const std::vector<T>& b, const char* what) {
    if (a.size() != b.size() || std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) != 0) {
        throw std::runtime_error(std::string("content differs: ") + what);
    }
}

void read_all(const std::string& src, const std::string& dir) {
    const Data x = load(src);
    same(bf::read_packed_voltage(dir + "/voltage.bin", x.d), x.volt, "voltage");
    same(bf::read_weights(dir + "/weights.bin", x.d), x.w, "weights");
    same(bf::read_tiled_weights(dir + "/tiled.bin", x.d), x.tw, "tiled weights");
    same(bf::read_quantized_intensities(dir + "/codes.bin", x.wd), x.codes, "codes");
    same(bf::read_quantization_parameters(dir + "/params.bin", x.wd), x.params, "parameters");
    const auto md = bf::read_quantized_output_metadata(dir + "/int8_meta.txt");
    if (md.output_dims.n_time != x.wd.n_time || md.output_dims.n_beams != x.c.B || md.input_n_time != x.c.T ||
        md.temporal_integration.integration_spectra != x.c.S || md.shard.shard_id != x.c.shard_id ||
        md.shard.absolute_frequency_start != x.shard.absolute_frequency_start ||
        md.shard.timestamp_start != x.c.ts_start || md.shard.timestamp_step != x.c.ts_step ||
        md.shard.loss_mask_id != x.c.loss_id || md.parameters_file != "params.bin") {
        throw std::runtime_error("int8 metadata fields differ");
    }
    const auto sh = bf::read_packed_shard(dir + "/shard_payload.bin", dir + "/shard_meta.txt",
                                          dir + "/shard_loss.bin", x.d);
    same(sh.payload, x.volt, "shard payload");
    same(sh.loss_mask, x.loss, "shard loss mask");
    if (sh.descriptor.shard_id != x.c.shard_id || sh.descriptor.timestamp_start != x.c.ts_start ||
        sh.descriptor.timestamp_step != x.c.ts_step || sh.descriptor.loss_mask_id != x.c.loss_id) {
        throw std::runtime_error("shard descriptor fields differ");
    }
    std::cout << "READ OK\n";
}

template <typename E, typename Fn>
void expect(const char* what, Fn&& fn) {
    try {
        fn();
    } catch (const E&) {
        return;
    } catch (const std::exception& e) {
        throw std::runtime_error(std::string(what) + ": wrong exception type: " + e.what());
    }
    throw std::runtime_error(std::string(what) + ": no exception");
}

void errors(const std::string& dir) {
    const bf::Dimensions d{4, 336, 32, 3};
    bf::PackedVoltage v(bf::voltage_sample_count(d), 0x11);
    bf::write_packed_voltage(dir + "/e_voltage.bin", v, d);
    // size mismatch on write: invalid_argument, nothing written
    expect<std::invalid_argument>("short voltage", [&] {
        bf::write_packed_voltage(dir + "/e_short.bin", bf::PackedVoltage(10), d);
    });
    expect<std::invalid_argument>("bad dims", [&] {
        bf::write_packed_voltage(dir + "/e_bad.bin", v, bf::Dimensions{4, 100, 32, 3});
    });
    // file-size check on read: runtime_error naming both sizes
    try {
        bf::read_packed_voltage(dir + "/e_voltage.bin", bf::Dimensions{5, 336, 32, 3});
        throw std::runtime_error("oversized read: no exception");
    } catch (const std::runtime_error& e) {
        const std::string m = e.what();
        if (m.find("43008 bytes; expected 53760") == std::string::npos) {
            throw std::runtime_error("file-size message: " + m);
        }
    }
    expect<std::runtime_error>("missing file", [&] { bf::read_weights(dir + "/no_such_file.bin", d); });
    // malformed metadata
    {
        std::ofstream bad(dir + "/e_meta.txt");
        bad << "format=beamformer-quantized-int8-v1\nno separator here\n";
    }
    expect<std::runtime_error>("malformed metadata", [&] { bf::read_quantized_output_metadata(dir + "/e_meta.txt"); });
    {
        std::ofstream bad(dir + "/e_meta2.txt");
        bad << "format=beamformer-quantized-int8-v2\n";
    }
    expect<std::runtime_error>("missing fields", [&] { bf::read_quantized_output_metadata(dir + "/e_meta2.txt"); });
    // invalid metadata on write: invalid_argument (time dimensions inconsistent)
    expect<std::invalid_argument>("inconsistent metadata", [&] {
        bf::write_quantized_output_metadata(
            dir + "/e_meta3.txt", bf::QuantizedOutputMetadata{bf::Dimensions{7, 336, 32, 3}, 4,
                                                              bf::TemporalIntegrationConfig{2},
                                                              bf::default_shard_descriptors()[0], "p.bin"});
    });
    // loss-mask values other than 0 / 1
    expect<std::invalid_argument>("loss mask value", [&] {
        bf::LossMask m(bf::loss_mask_count(d), 1);
        m[3] = 2;
        bf::write_packed_shard(dir + "/e_p.bin", dir + "/e_m.txt", dir + "/e_l.bin",
                               bf::PackedShard{bf::default_shard_descriptors()[0], v, m}, d);
    });
    // shard metadata whose dimensions disagree with the caller's
    {
        bf::LossMask m(bf::loss_mask_count(d), 1);
        bf::write_packed_shard(dir + "/e_p.bin", dir + "/e_m.txt", dir + "/e_l.bin",
                               bf::PackedShard{bf::default_shard_descriptors()[1], v, m}, d);
    }
    expect<std::runtime_error>("shard dims", [&] {
        bf::read_packed_shard(dir + "/e_p.bin", dir + "/e_m.txt", dir + "/e_l.bin", bf::Dimensions{4, 336, 32, 4});
    });
    std::cout << "ERRORS OK\n";
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "write" && argc == 4) write_all(argv[2], argv[3]);
        else if (mode == "read" && argc == 4) read_all(argv[2], argv[3]);
        else if (mode == "errors" && argc == 3) errors(argv[2]);
        else {
            std::cerr << "usage: test_io write SRC OUT | read SRC DIR | errors DIR\n";
            return 2;
        }
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "FAIL: " << e.what() << "\n";
        return 1;
    }
}
