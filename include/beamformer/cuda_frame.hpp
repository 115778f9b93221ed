// cuda_frame.hpp -- non-owning device frame views.  Same declarations and
// validation rules as the reference's include/beamformer/cuda_frame.hpp:
// 14-231 (a typed, shaped device buffer plus frame id and shard metadata),
// used by CudaBeamformerWorkspace::run_device_frame.
#pragma once

#include "beamformer/config.hpp"
#include "beamformer/formats.hpp"
#include "beamformer/quantization.hpp"

#include <array>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>

namespace beamformer {

inline constexpr std::size_t cuda_frame_max_rank = 4;
using FrameShape = std::array<std::size_t, cuda_frame_max_rank>;

enum class CudaDataType {
    PackedInt4x2,
    ComplexFloat32,
    Float32,
    SignedInt8,
};

constexpr std::size_t cuda_data_type_size(const CudaDataType type) {
    switch (type) {
        case CudaDataType::PackedInt4x2:
        case CudaDataType::SignedInt8:
            return 1;
        case CudaDataType::ComplexFloat32:
            return 8;
        case CudaDataType::Float32:
            return 4;
    }
    return 0;
}

struct CudaBufferView {
    void* device_data = nullptr;
    std::size_t bytes = 0;
    CudaDataType type = CudaDataType::Float32;
    std::size_t rank = 0;
    FrameShape shape{};
    FrameShape strides_bytes{};  // in bytes
};

struct CudaFrameMetadata {
    std::uint64_t frame_id = 0;
    ShardDescriptor shard;
};

struct CudaFrameView {
    CudaBufferView buffer;
    CudaFrameMetadata metadata;
};

inline std::size_t cuda_frame_element_count(const FrameShape& shape, const std::size_t rank) {
    if (rank == 0 || rank > cuda_frame_max_rank) throw std::invalid_argument("CUDA frame rank must be between 1 and 4");
    std::size_t count = 1;
    for (std::size_t axis = 0; axis < rank; ++axis) {
        if (shape[axis] == 0 || count > std::numeric_limits<std::size_t>::max() / shape[axis]) {
            throw std::invalid_argument("CUDA frame shape is empty or overflows size_t");
        }
        count *= shape[axis];
    }
    for (std::size_t axis = rank; axis < cuda_frame_max_rank; ++axis) {
        if (shape[axis] != 0) throw std::invalid_argument("unused CUDA frame shape axes must be zero");
    }
    return count;
}

inline FrameShape cuda_contiguous_strides_bytes(const CudaDataType type, const FrameShape& shape,
                                                const std::size_t rank) {
    cuda_frame_element_count(shape, rank);
    FrameShape strides{};
    std::size_t stride = cuda_data_type_size(type);
    for (std::size_t axis = rank; axis-- > 0;) {
        strides[axis] = stride;
        if (shape[axis] > std::numeric_limits<std::size_t>::max() / stride) {
            throw std::invalid_argument("CUDA frame strides overflow size_t");
        }
        stride *= shape[axis];
    }
    return strides;
}

// Bytes spanned from the first element to the end of the last one.
inline std::size_t cuda_frame_minimum_storage_bytes(const CudaBufferView& b) {
    if (b.rank == 0 || b.rank > cuda_frame_max_rank) throw std::invalid_argument("CUDA buffer rank must be between 1 and 4");
    cuda_frame_element_count(b.shape, b.rank);
    std::size_t end = cuda_data_type_size(b.type);
    for (std::size_t axis = 0; axis < b.rank; ++axis) {
        if (b.strides_bytes[axis] == 0) throw std::invalid_argument("CUDA buffer strides must be positive");
        const std::size_t extent = b.shape[axis] - 1;
        if (extent > (std::numeric_limits<std::size_t>::max() - end) / b.strides_bytes[axis]) {
            throw std::invalid_argument("CUDA buffer storage size overflows size_t");
        }
        end += extent * b.strides_bytes[axis];
    }
    for (std::size_t axis = b.rank; axis < cuda_frame_max_rank; ++axis) {
        if (b.strides_bytes[axis] != 0) throw std::invalid_argument("unused CUDA buffer strides must be zero");
    }
    return end;
}

inline bool cuda_buffer_view_is_contiguous(const CudaBufferView& b) {
    return b.strides_bytes == cuda_contiguous_strides_bytes(b.type, b.shape, b.rank);
}

inline void validate_cuda_buffer_view(const CudaBufferView& b) {
    if (b.device_data == nullptr) throw std::invalid_argument("CUDA buffer device_data must not be null");
    if (b.bytes < cuda_frame_minimum_storage_bytes(b)) {
        throw std::invalid_argument("CUDA buffer bytes are smaller than its shape and strides");
    }
}

inline void validate_contiguous_cuda_buffer_view(const CudaBufferView& b) {
    validate_cuda_buffer_view(b);
    if (!cuda_buffer_view_is_contiguous(b)) throw std::invalid_argument("CUDA frame must use contiguous storage");
}

inline CudaFrameView make_contiguous_cuda_frame_view(void* device_data, std::size_t bytes, CudaDataType type,
                                                     const FrameShape& shape, std::size_t rank,
                                                     std::uint64_t frame_id, const ShardDescriptor& shard) {
    validate_shard_descriptor(shard);
    CudaFrameView f;
    f.buffer.device_data = device_data;
    f.buffer.bytes = bytes;
    f.buffer.type = type;
    f.buffer.rank = rank;
    f.buffer.shape = shape;
    f.buffer.strides_bytes = cuda_contiguous_strides_bytes(type, shape, rank);
    f.metadata.frame_id = frame_id;
    f.metadata.shard = shard;
    validate_contiguous_cuda_buffer_view(f.buffer);
    return f;
}

inline CudaFrameView make_packed_voltage_frame_view(void* p, const Dimensions& d, std::uint64_t id,
                                                    const ShardDescriptor& s) {
    validate_dimensions(d);
    return make_contiguous_cuda_frame_view(p, packed_voltage_bytes(d), CudaDataType::PackedInt4x2,
                                           {d.n_time, d.n_freq, d.n_ant, 0}, 3, id, s);
}

inline CudaFrameView make_intensity_frame_view(void* p, const Dimensions& d, std::uint64_t id,
                                               const ShardDescriptor& s) {
    validate_dimensions(d);
    return make_contiguous_cuda_frame_view(p, intensity_bytes(d), CudaDataType::Float32,
                                           {d.n_time, d.n_freq, d.n_beams, 0}, 3, id, s);
}

inline CudaFrameView make_quantized_intensity_frame_view(void* p, const Dimensions& d, std::uint64_t id,
                                                         const ShardDescriptor& s) {
    validate_dimensions(d);
    return make_contiguous_cuda_frame_view(p, quantized_intensity_bytes(d), CudaDataType::SignedInt8,
                                           {d.n_time, d.n_freq, d.n_beams, 0}, 3, id, s);
}

inline CudaFrameView make_weights_frame_view(void* p, const Dimensions& d, std::uint64_t id,
                                             const ShardDescriptor& s) {
    validate_dimensions(d);
    return make_contiguous_cuda_frame_view(p, weight_bytes(d), CudaDataType::ComplexFloat32,
                                           {d.n_beams, d.n_freq, d.n_ant, 0}, 3, id, s);
}

inline CudaFrameView make_tiled_weights_frame_view(void* p, const Dimensions& d, std::uint64_t id,
                                                   const ShardDescriptor& s) {
    validate_dimensions(d);
    return make_contiguous_cuda_frame_view(p, tiled_weight_bytes(d), CudaDataType::ComplexFloat32,
                                           {d.n_freq, tiled_weight_beam_tiles(d), d.n_ant, tiled_weight_beam_tile},
                                           4, id, s);
}

inline CudaFrameView make_quantization_parameters_frame_view(void* p, const Dimensions& integrated_dims,
                                                             std::uint64_t id, const ShardDescriptor& s) {
    validate_dimensions(integrated_dims);
    const auto l = quantization_layout(integrated_dims);
    return make_contiguous_cuda_frame_view(p, quantization_parameter_count(integrated_dims) * 2 * sizeof(float),
                                           CudaDataType::Float32, {l.time_tiles, l.frequency_tiles, l.beam_tiles, 2},
                                           4, id, s);
}

inline void validate_cuda_frame_view(const CudaFrameView& frame) {
    validate_cuda_buffer_view(frame.buffer);
    validate_shard_descriptor(frame.metadata.shard);
}

}  // namespace beamformer
