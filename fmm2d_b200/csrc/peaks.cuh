// Arithmetic-pipe throughput microbenchmark (roofline denominators for the
// FMA-bound near-field kernels).
#pragma once

namespace b2 {
double fma_peak_flops(bool fp64);
}
