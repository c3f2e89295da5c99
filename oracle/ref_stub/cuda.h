#pragma once
#include "cuda_host_shim.h"
