// cvl_internal.h -- what the host-side translation units of libcvl share
// beyond the public C ABI.
#pragma once

#include <cstdint>
#include <string>

#include "../../include/cvl.h"

// Records msg as the calling thread's cvl_last_error() and returns code.
int cvl_fail(int code, const std::string &msg);

struct cvl_engine;

// A host hook that the engine calls between the bundle/growth chunks of a run,
// once the previous chunk's kernels have finished. The hook may block to let
// other streams' work through first (the server uses it to yield a large map
// to small ones); nullptr removes it.
using cvl_yield_fn = void (*)(void *ctx);
void cvl_engine_set_yield(cvl_engine *e, cvl_yield_fn fn, void *ctx);

// Sets aside `bytes` of page-locked host memory in the engine's result arena
// (one chunk made ahead of time, so results do not pin memory while serving).
int cvl_engine_reserve_host(cvl_engine *e, size_t bytes);

// Maps `bytes` of device memory into the engine's memory pool ahead of time (an
// allocation freed at once: the pool keeps what it has), so that later workspace
// growth is carved from memory already mapped.
int cvl_engine_reserve_device(cvl_engine *e, size_t bytes);

// An empty device batch of the engine with room for max_edges rows of
// edge_data_sz values in up to max_maps maps, allocated now: refills within
// that size reuse it.
struct cvl_batch;
int cvl_batch_create_reserved(cvl_engine *e, int64_t max_edges, int32_t max_maps, int32_t edge_data_sz,
                              cvl_batch **out);

// cvl_engine_workspace_bytes for an engine with this tuning per bucket (no record
// arena of past inputs counted): the footprint of a launch of that shape.
int cvl_workspace_bytes_tuned(const cvl_tuning *tune, const cvl_workspace_shape *s, const cvl_params *p,
                              size_t *total, size_t *per_launch);

// Growth of the engine's memory so far: device workspace allocations (calls that
// allocated from the engine's pool) and page-locked result chunks, with the host
// time the calls took.
void cvl_engine_growth(const cvl_engine *e, uint64_t *dev_grows, double *dev_ms, uint64_t *host_grows,
                       double *host_ms);
