// Stand-in for Daxa's task-graph declaration macros (parity oracle only).
// Task heads describe Vulkan resource usage for the editing passes, which
// the oracle never runs.
#pragma once
#define DAXA_DECL_TASK_HEAD_BEGIN(NAME)
#define DAXA_TH_BUFFER_PTR(...)
#define DAXA_DECL_TASK_HEAD_END
#define DAXA_TH_BLOB(HEAD, NAME) int NAME;
