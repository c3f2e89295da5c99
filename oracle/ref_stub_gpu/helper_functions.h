/* Stand-in for the CUDA-samples helper header the reference includes (nothing of it is used). */
#pragma once
