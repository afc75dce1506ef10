// Stub used only by the host build of the reference kernels (oracle/_ref).
#pragma once
namespace cooperative_groups {
struct thread_block { void sync() {} };
inline thread_block this_thread_block() { return {}; }
}
