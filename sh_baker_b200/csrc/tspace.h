// tspace.h - per-vertex tangent frames for meshes that carry no TANGENT
// attribute (the reference's GenerateTangents, src/loader.cpp:88-109).
#pragma once

#include <cstddef>
#include <cstdint>

namespace shb {

// Writes 4 floats per vertex (tangent xyz, handedness sign) into `out` for
// the triangle list `idx` over `nv` vertices with positions `pos` (3 per
// vertex), normals `nrm` (3) and texture UVs `uv` (2).  Vertices that no
// triangle defines a tangent for keep the reference's geometric fallback
// (src/loader.cpp:370-385).
void generate_tangent_frames(const float* pos, const float* nrm, const float* uv, size_t nv, const uint32_t* idx,
                             size_t n_idx, float* out);

}  // namespace shb
