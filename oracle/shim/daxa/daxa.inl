// Stand-in for Daxa's daxa/daxa.inl when the cube-tracing shaders are
// compiled as C++ by the parity oracle (test infrastructure only).
#pragma once
#include "../glsl_shim.hpp"
