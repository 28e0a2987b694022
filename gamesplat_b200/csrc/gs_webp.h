// Lossless WebP decoding for the SOG loader (host code).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/gs_api.h"

namespace gs {

// Decodes a lossless WebP image (RIFF container or raw VP8L bitstream) to
// RGBA8, rows top first.  With rgba == nullptr only the size is read.
// Returns false for lossy, animated or invalid images.
bool webp_decode_rgba(const uint8_t* data, size_t size, int* width, int* height, std::vector<uint8_t>* rgba);

}  // namespace gs
