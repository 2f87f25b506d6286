// rcp64_check.cu -- accuracy check of the FP64 reciprocal the RHS kernels use (abl::rcp64 in
// ablate_b200/csrc/fv_physics.cuh) against the IEEE division 1/x computed on the host.
//
// Reads doubles from stdin-free generated inputs (the host builds them: log-uniform magnitudes over the
// whole exponent range, both signs, the approximation's cut-offs 1e-300 and 1e300 with their neighbours,
// powers of two, mantissa extremes, zeros, subnormals, infinities and NaN), evaluates rcp64 on the
// device, and prints one line: "n <count> max_ulp <worst error against the exact 1/x, in units of the last
// place of the correctly rounded 1/x> not_nearest <results that are the neighbour of the correctly rounded
// value> mismatched_specials <count>". The error against the exact reciprocal comes from the residual
// 1 - x y, which one fused multiply-add computes exactly when y is within a few ulps of 1/x.
// Built and run by tests/test_rcp64.py.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../ablate_b200/csrc/fv_physics.cuh"

__global__ void k_rcp(const double* x, double* y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = abl::rcp64(x[i]);
}

static double ulp_of(double v) {
    v = std::fabs(v);
    const double next = std::nextafter(v, INFINITY);
    return next - v;
}

int main() {
    std::vector<double> x;
    std::mt19937_64 rng(20261203);
    std::uniform_real_distribution<double> e10(-307.0, 307.0), u01(1.0, 2.0);
    for (int i = 0; i < 2000000; i++) {
        const double m = std::pow(10.0, e10(rng));
        x.push_back((i & 1) ? -m : m);
    }
    for (int i = 0; i < 500000; i++) x.push_back(u01(rng) * ((i & 1) ? -1.0 : 1.0));  // dense mantissas in one binade
    for (double t : {1e-300, 1e300}) {
        double lo = t, hi = t;
        for (int k = 0; k < 64; k++) {
            x.push_back(lo);
            x.push_back(-lo);
            x.push_back(hi);
            x.push_back(-hi);
            lo = std::nextafter(lo, 0.0);
            hi = std::nextafter(hi, INFINITY);
        }
    }
    for (int e = -1074; e <= 1023; e++) {
        const double p = std::ldexp(1.0, e);
        x.push_back(p);
        x.push_back(-p);
        x.push_back(std::nextafter(p, INFINITY));
        x.push_back(std::nextafter(2 * p, 0.0));
    }
    const double specials[] = {0.0, -0.0, INFINITY, -INFINITY, NAN, 4.9e-324, -4.9e-324, 2.2250738585072014e-308, 1.7976931348623157e308};
    for (double s : specials) x.push_back(s);
    const int n = (int)x.size();
    double *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, n * sizeof(double)) != cudaSuccess || cudaMalloc(&dy, n * sizeof(double)) != cudaSuccess) {
        std::printf("error cudaMalloc\n");
        return 2;
    }
    cudaMemcpy(dx, x.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    k_rcp<<<(n + 255) / 256, 256>>>(dx, dy, n);
    std::vector<double> y(n);
    if (cudaMemcpy(y.data(), dy, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        std::printf("error kernel\n");
        return 2;
    }
    double worst = 0.0;
    long bad_special = 0, not_nearest = 0;
    for (int i = 0; i < n; i++) {
        const double ref = 1.0 / x[i];
        if (!std::isfinite(ref) || ref == 0.0 || std::fpclassify(ref) == FP_SUBNORMAL) {
            // zero, infinite, NaN and subnormal results: the exact IEEE value (sign included)
            const bool same = (std::isnan(ref) && std::isnan(y[i])) || (std::memcmp(&ref, &y[i], sizeof(double)) == 0);
            if (!same) bad_special++;
            continue;
        }
        if (y[i] != ref) not_nearest++;
        // |1/x - y| = |1 - x y| / |x|, the residual exact by one rounding of the fused multiply-add
        const double err = std::fabs(std::fma(-x[i], y[i], 1.0)) / std::fabs(x[i]) / ulp_of(ref);
        if (!(err <= worst)) worst = std::isnan(err) ? INFINITY : err;
    }
    cudaFree(dx);
    cudaFree(dy);
    std::printf("n %d max_ulp %.6g not_nearest %ld mismatched_specials %ld\n", n, worst, not_nearest, bad_special);
    return 0;
}
