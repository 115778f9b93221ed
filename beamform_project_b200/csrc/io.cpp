// io.cpp -- the on-disk formats of include/beamformer/io.hpp.
//
// The byte layouts and the two key=value metadata formats are the
// reference's (src/io.cpp:60-344): files written here and there are
// identical, and each side reads the other's.  Binary arrays go through one
// checked reader and writer; metadata goes through an ordered key=value
// writer and a parser that keeps the last value of a repeated key.
#include "beamformer/io.hpp"

#include <cstdint>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <system_error>
#include <utility>
#include <vector>

namespace beamformer {
namespace {

namespace fs = std::filesystem;

template <typename T>
std::vector<T> load_array(const fs::path& path, std::size_t count) {
    std::error_code ec;
    const std::uintmax_t size = fs::file_size(path, ec);
    if (ec) throw std::runtime_error("cannot inspect input file: " + path.string());
    const std::uintmax_t want = static_cast<std::uintmax_t>(count) * sizeof(T);
    if (size != want) {
        throw std::runtime_error(path.string() + " has " + std::to_string(size) + " bytes; expected " +
                                 std::to_string(want));
    }
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open input file: " + path.string());
    std::vector<T> data(count);
    in.read(reinterpret_cast<char*>(data.data()), static_cast<std::streamsize>(want));
    if (!in) throw std::runtime_error("failed to read input file: " + path.string());
    return data;
}

template <typename T>
void store_array(const fs::path& path, const std::vector<T>& data) {
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) throw std::runtime_error("cannot open output file: " + path.string());
    out.write(reinterpret_cast<const char*>(data.data()), static_cast<std::streamsize>(data.size() * sizeof(T)));
    if (!out) throw std::runtime_error("failed to write output file: " + path.string());
}

template <typename T>
void require_count(const std::vector<T>& data, std::size_t count, const char* what) {
    if (data.size() != count) throw std::invalid_argument(std::string(what) + " does not match dimensions");
}

using Fields = std::vector<std::pair<std::string, std::string>>;

void store_fields(const fs::path& path, const Fields& fields, const char* what) {
    std::ofstream out(path, std::ios::trunc);
    if (!out) throw std::runtime_error(std::string("cannot open ") + what + " file: " + path.string());
    for (const auto& kv : fields) out << kv.first << '=' << kv.second << '\n';
    if (!out) throw std::runtime_error(std::string("failed to write ") + what + " file: " + path.string());
}

// key=value lines; a line without '=' or with an empty key is an error
class FieldMap {
public:
    FieldMap(const fs::path& path, const char* what) : path_(path), what_(what) {
        std::ifstream in(path);
        if (!in) throw std::runtime_error(std::string("cannot open ") + what + " file: " + path.string());
        std::string line;
        while (std::getline(in, line)) {
            const std::size_t eq = line.find('=');
            if (eq == std::string::npos || eq == 0) {
                throw std::runtime_error(std::string("invalid ") + what + " line in: " + path.string());
            }
            fields_[line.substr(0, eq)] = line.substr(eq + 1);
        }
    }
    const std::string& text(const char* key) const {
        const auto it = fields_.find(key);
        if (it == fields_.end()) {
            throw std::runtime_error(std::string("missing ") + what_ + " field " + key + " in: " + path_.string());
        }
        return it->second;
    }
    std::size_t size(const char* key) const { return static_cast<std::size_t>(std::stoull(text(key))); }
    std::uint64_t u64(const char* key) const { return static_cast<std::uint64_t>(std::stoull(text(key))); }
    bool flag(const char* key) const {
        const std::string& v = text(key);
        if (v != "0" && v != "1") throw std::runtime_error(std::string("invalid ") + what_ + " flag " + key);
        return v == "1";
    }

private:
    fs::path path_;
    const char* what_;
    std::map<std::string, std::string> fields_;
};

void add(Fields& f, const char* key, const std::string& value) { f.emplace_back(key, value); }
void add(Fields& f, const char* key, std::uint64_t value) { f.emplace_back(key, std::to_string(value)); }

void add_shard(Fields& f, const ShardDescriptor& d) {
    add(f, "shard_id", d.shard_id);
    add(f, "shard_count", d.shard_count);
    add(f, "local_frequency_count", d.local_frequency_count);
    add(f, "absolute_frequency_start", d.absolute_frequency_start);
    add(f, "timestamp_start", d.timestamp_start);
    add(f, "timestamp_step", d.timestamp_step);
    add(f, "loss_mask_id", d.loss_mask_id);
    add(f, "loss_mask_independent", std::uint64_t{d.loss_mask_independent ? 1u : 0u});
}

ShardDescriptor read_shard(const FieldMap& m) {
    ShardDescriptor d;
    d.shard_id = m.size("shard_id");
    d.shard_count = m.size("shard_count");
    d.local_frequency_count = m.size("local_frequency_count");
    d.absolute_frequency_start = m.size("absolute_frequency_start");
    d.timestamp_start = m.u64("timestamp_start");
    d.timestamp_step = m.u64("timestamp_step");
    d.loss_mask_id = m.u64("loss_mask_id");
    d.loss_mask_independent = m.flag("loss_mask_independent");
    return d;
}

constexpr const char* kShardFormat = "beamformer-packed-shard-v1";
constexpr const char* kInt8Format = "beamformer-quantized-int8-v1";
constexpr const char* kParamsFormat = "little-endian-float32[offset,scale]";

}  // namespace

PackedVoltage read_packed_voltage(const fs::path& path, const Dimensions& dims) {
    validate_dimensions(dims);
    return load_array<std::uint8_t>(path, voltage_sample_count(dims));
}

void write_packed_voltage(const fs::path& path, const PackedVoltage& voltage, const Dimensions& dims) {
    validate_dimensions(dims);
    require_count(voltage, voltage_sample_count(dims), "packed voltage size");
    store_array(path, voltage);
}

Weights read_weights(const fs::path& path, const Dimensions& dims) {
    validate_dimensions(dims);
    return load_array<ComplexFloat>(path, dims.n_beams * dims.n_freq * dims.n_ant);
}

void write_weights(const fs::path& path, const Weights& weights, const Dimensions& dims) {
    validate_dimensions(dims);
    require_count(weights, dims.n_beams * dims.n_freq * dims.n_ant, "weight count");
    store_array(path, weights);
}

TiledWeights read_tiled_weights(const fs::path& path, const Dimensions& dims) {
    validate_dimensions(dims);
    return load_array<ComplexFloat>(path, tiled_weight_count(dims));
}

void write_tiled_weights(const fs::path& path, const TiledWeights& weights, const Dimensions& dims) {
    validate_dimensions(dims);
    require_count(weights, tiled_weight_count(dims), "tiled weight count");
    store_array(path, weights);
}

void write_intensities(const fs::path& path, const Intensities& intensities, const Dimensions& dims) {
    validate_dimensions(dims);
    require_count(intensities, dims.n_time * dims.n_freq * dims.n_beams, "intensity count");
    store_array(path, intensities);
}

QuantizedIntensities read_quantized_intensities(const fs::path& path, const Dimensions& dims) {
    validate_dimensions(dims);
    return load_array<std::int8_t>(path, dims.n_time * dims.n_freq * dims.n_beams);
}

void write_quantized_intensities(const fs::path& path, const QuantizedIntensities& intensities,
                                 const Dimensions& dims) {
    validate_dimensions(dims);
    require_count(intensities, dims.n_time * dims.n_freq * dims.n_beams, "quantized intensity count");
    store_array(path, intensities);
}

std::vector<Int8QuantizationParameters> read_quantization_parameters(const fs::path& path,
                                                                     const Dimensions& integrated_dims) {
    return load_array<Int8QuantizationParameters>(path, quantization_parameter_count(integrated_dims));
}

void write_quantization_parameters(const fs::path& path, const std::vector<Int8QuantizationParameters>& parameters,
                                   const Dimensions& integrated_dims) {
    require_count(parameters, quantization_parameter_count(integrated_dims), "quantization parameter count");
    store_array(path, parameters);
}

void write_quantized_output_metadata(const fs::path& path, const QuantizedOutputMetadata& metadata) {
    validate_quantized_output_metadata(metadata);
    const Dimensions& d = metadata.output_dims;
    Fields f;
    add(f, "format", kInt8Format);
    add(f, "n_time", d.n_time);
    add(f, "n_freq", d.n_freq);
    add(f, "n_ant", d.n_ant);
    add(f, "n_beams", d.n_beams);
    add(f, "input_n_time", metadata.input_n_time);
    add(f, "integration_spectra", metadata.temporal_integration.integration_spectra);
    add(f, "chunk_time", quantization_chunk_time);
    add(f, "chunk_frequency", quantization_chunk_frequency);
    add(f, "chunk_beam", quantization_chunk_beam);
    add(f, "invalid_code", std::to_string(static_cast<int>(quantized_invalid_code)));
    add(f, "parameters_format", kParamsFormat);
    add(f, "parameters_file", metadata.parameters_file);
    add(f, "parameters_count", quantization_parameter_count(d));
    add_shard(f, metadata.shard);
    store_fields(path, f, "quantized metadata");
}

QuantizedOutputMetadata read_quantized_output_metadata(const fs::path& path) {
    const FieldMap m(path, "quantized metadata");
    if (m.text("format") != kInt8Format || m.text("parameters_format") != kParamsFormat ||
        m.size("chunk_time") != quantization_chunk_time || m.size("chunk_frequency") != quantization_chunk_frequency ||
        m.size("chunk_beam") != quantization_chunk_beam ||
        std::stoi(m.text("invalid_code")) != quantized_invalid_code) {
        throw std::runtime_error("unsupported quantized metadata format: " + path.string());
    }
    QuantizedOutputMetadata md;
    md.output_dims = Dimensions{m.size("n_time"), m.size("n_freq"), m.size("n_ant"), m.size("n_beams")};
    md.input_n_time = m.size("input_n_time");
    md.temporal_integration = TemporalIntegrationConfig{m.size("integration_spectra")};
    md.shard = read_shard(m);
    md.parameters_file = m.text("parameters_file");
    if (m.size("parameters_count") != quantization_parameter_count(md.output_dims)) {
        throw std::runtime_error("quantization parameter count is inconsistent: " + path.string());
    }
    validate_quantized_output_metadata(md);
    return md;
}

void write_packed_shard(const fs::path& payload_path, const fs::path& metadata_path, const fs::path& loss_mask_path,
                        const PackedShard& shard, const Dimensions& dims) {
    validate_packed_shard(shard, dims);
    write_packed_voltage(payload_path, shard.payload, dims);
    store_array(loss_mask_path, shard.loss_mask);
    Fields f;
    add(f, "format", kShardFormat);
    add(f, "n_time", dims.n_time);
    add(f, "n_freq", dims.n_freq);
    add(f, "n_ant", dims.n_ant);
    add(f, "n_beams", dims.n_beams);
    add_shard(f, shard.descriptor);
    add(f, "payload_bytes", shard.payload.size());
    add(f, "loss_mask_bytes", shard.loss_mask.size());
    store_fields(metadata_path, f, "shard metadata");
}

PackedShard read_packed_shard(const fs::path& payload_path, const fs::path& metadata_path,
                              const fs::path& loss_mask_path, const Dimensions& dims) {
    validate_dimensions(dims);
    const FieldMap m(metadata_path, "shard metadata");
    if (m.text("format") != kShardFormat || m.size("n_time") != dims.n_time || m.size("n_freq") != dims.n_freq ||
        m.size("n_ant") != dims.n_ant || m.size("n_beams") != dims.n_beams ||
        m.size("payload_bytes") != packed_voltage_bytes(dims) || m.size("loss_mask_bytes") != loss_mask_count(dims)) {
        throw std::runtime_error("shard metadata does not match dimensions: " + metadata_path.string());
    }
    PackedShard shard;
    shard.descriptor = read_shard(m);
    shard.payload = read_packed_voltage(payload_path, dims);
    shard.loss_mask = load_array<std::uint8_t>(loss_mask_path, loss_mask_count(dims));
    validate_packed_shard(shard, dims);
    return shard;
}

}  // namespace beamformer
