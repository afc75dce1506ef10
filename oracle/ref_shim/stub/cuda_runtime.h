// Stub used only by the host build of the reference kernels (oracle/_ref):
// the kernels are compiled as host code and call no CUDA runtime function.
#pragma once
