// fv_consts.hpp -- constants shared by the host-side set-up and the device kernels.
#pragma once

// Loops over the components of a state row (species-sized) are unrolled, except in the translation
// units of the species-capacity instances (ABL_CAPACITY_TU), which serve any species count up to
// kMaxSpecies through run-time loops: unrolled, their rows of up to 133 components do not compile in
// reasonable time. Loops over the dimension stay unrolled everywhere.
#ifdef ABL_CAPACITY_TU
#define ABL_UNROLL_SPECIES _Pragma("unroll 1")
#else
#define ABL_UNROLL_SPECIES _Pragma("unroll")
#endif

// The loops of the NASA-7 mixture functions (the mass fractions, e_s, cp, the molar mass) follow the
// species loops, except in the unit of the 64-species tangent (ABL_CAPACITY_UNROLL_MIXTURE), which
// keeps them unrolled: built with those loops at run time, the capacity instances' tangent kernels
// returned NaN where their RHS was exact, and unrolled at 64 species they compile in minutes.
#if defined(ABL_CAPACITY_TU) && !defined(ABL_CAPACITY_UNROLL_MIXTURE)
#define ABL_UNROLL_MIXTURE _Pragma("unroll 1")
#else
#define ABL_UNROLL_MIXTURE _Pragma("unroll")
#endif

namespace abl {

// Faces per colour in a tile (the adjoint kernel runs one colour per pass, two lanes per face, on
// 2 * kColorCap threads).
constexpr int kColorCap = 128;

// Largest species count a physics descriptor may carry (the per-thread scratch of the EOS batch
// kernels is sized by it; the largest capacity instance holds it).
constexpr int kMaxSpecies = 128;

// Instances compiled with their flux calculator and limiter fixed at compile time (and the fused
// kernel, the adjoint and the stepping kernels): the exact species counts up to 9. The 16-species
// instances (RHS, aux update, tangent) and the kMaxSpecies capacity instances (RHS and aux update, run-
// time loops) run the generic kernels only.
template <int NS>
constexpr bool kSpecialized = NS <= 9;

}  // namespace abl
