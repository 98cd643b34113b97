// TEST INFRASTRUCTURE ONLY -- stand-in for the CMake-generated
// barneyDeviceConfig.h of the reference's CPU backend: the compiled reference
// files live in namespace barney_cpu, single-scatter build.
#pragma once
#define BARNEY_NS barney_cpu
#define BARNEY_BACKEND_CPU 1
#define BARNEY_HAVE_CUDA 0
#define BARNEY_MPI 0
#define BARNEY_USE_MULTI_SCATTERING 0
#define BARNEY_DISABLE_DENOISING 1
