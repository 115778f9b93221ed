// int4.hpp -- kept for source compatibility with callers of the reference's
// include/beamformer/int4.hpp; the declarations live in formats.hpp.
#pragma once

#include "beamformer/formats.hpp"
