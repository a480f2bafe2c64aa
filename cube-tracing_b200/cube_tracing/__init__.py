"""B200 hot path of cube-tracing: voxel ray tracing, ReSTIR DI and TAA behind
the C ABI of include/ct.h (libct.so in this directory)."""
