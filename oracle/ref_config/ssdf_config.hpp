// Configuration header for compiling the reference's CPU sources directly with g++ (oracle/Makefile),
// standing in for the one its CMake build would generate: OpenMP on, no MPI, no CUDA/HIP, no cuBQL.
#ifndef SSDF_CONFIG_HPP
#define SSDF_CONFIG_HPP
#define SSDF_VERSION "reference-cpu"
#define SSDF_ENABLE_OPENMP
#endif
