// kernels_pow2.cu -- the kernels for grids whose FFT length M = NP/2 is a power of two.
#define SDFT_FFT_GEN 0
#include "kernels.cuh"
