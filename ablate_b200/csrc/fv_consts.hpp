// fv_consts.hpp -- constants shared by the host-side set-up and the device kernels.
#pragma once

namespace abl {

// Faces per colour in a tile (the adjoint kernel runs one colour per pass, two lanes per face, on
// 2 * kColorCap threads).
constexpr int kColorCap = 128;

// Largest species count a physics descriptor may carry (the per-thread scratch of the EOS batch
// kernels is sized by it).
constexpr int kMaxSpecies = 128;

}  // namespace abl
