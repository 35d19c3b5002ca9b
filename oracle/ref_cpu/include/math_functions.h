// ORACLE -- test infrastructure only.
// Stands in for the CUDA header of this name under the host execution model.
#pragma once
#include "cuda_runtime.h"
