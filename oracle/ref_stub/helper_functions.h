/* Stand-in for the CUDA-samples helper header; the reference uses nothing from it. */
#pragma once
