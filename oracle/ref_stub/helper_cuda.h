/* Stand-in for the CUDA-samples helper header that the reference includes.
   Only checkCudaErrors is used by the reference sources compiled here. */
#pragma once
#include <cstdio>
#include <cstdlib>
#define checkCudaErrors(val) do { if ((int)(val) != 0) { std::fprintf(stderr, "cuda error %d\n", (int)(val)); std::exit(1); } } while (0)
