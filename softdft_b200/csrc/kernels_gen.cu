// kernels_gen.cu -- the kernels for grids whose FFT length M = NP/2 is not a power of two.
#define SDFT_FFT_GEN 1
#include "kernels.cuh"
