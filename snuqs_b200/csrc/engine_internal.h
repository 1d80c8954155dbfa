// Library-internal hooks between the engine (engine.cu) and the other
// translation units of libsnuqs_b200.so.  Not part of the C ABI.
#pragma once
#include <stddef.h>

struct sq_state;

// Records `msg` for sq_last_error() and returns `code`.
int sq_detail_fail(int code, const char *msg);
// A device buffer of at least `bytes` owned by the state (grow-only, freed
// with the state) for result kernels' scratch.  Calls on one state that
// overlap on the GPU share it: order them on one stream.
int sq_detail_state_scratch(sq_state *s, size_t bytes, void **out);
// A pinned host buffer of at least `bytes` owned by the state (grow-only,
// freed with the state): staging for results copied to or from host buffers.
int sq_detail_state_host_scratch(sq_state *s, size_t bytes, void **out);
