// complex.hpp -- kept for source compatibility with callers of the reference's
// include/beamformer/complex.hpp; the declarations live in formats.hpp.
#pragma once

#include "beamformer/formats.hpp"
