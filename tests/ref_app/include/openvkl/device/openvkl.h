/* Stand-in for the reference's <openvkl/device/openvkl.h> (the CPU device's
 * sampling and iterator entry points); openvkl_cuda.h declares them. */
#pragma once
#include "../openvkl.h"
