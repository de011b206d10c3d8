/* Stand-in for the reference's <openvkl/openvkl.h> when an unchanged Open VKL
 * application is built against the cuda device (tests/ref_app/Makefile): the
 * cuda device's header declares the same API.  The application asks for the
 * reference's "cpu" device by name; built this way it gets the cuda device. */
#pragma once
#include "openvkl_cuda.h"
#define vklNewDevice(deviceName) vklNewDevice("cuda")
