// CUDA-graph replay of the solver loops' steps: one stream, no host synchronisation inside a step.
//
// The loops of calc_direct and calc_adjoint (computation_direct.f90:64-107,
// computation_adjoint.f90:60-108) repeat the same launches every step with the same buffers; only the
// filter pattern (which filters are due at step nt) changes.  A cache lives for one run call, keyed
// by the step's kind (loop and filter pattern) and its buffer pointers: the first sighting of a key
// runs eagerly (lazy allocations and one-time host reads such as the FP32 offsets happen there), the
// second records the step on the context's stream and instantiates it, later ones launch the graph.
// Because a cache never outlives the call, nothing a setter changes between calls (forcing, closure,
// adjoint mode, reference state) can go stale inside a graph.
#include "cruna_internal.cuh"

namespace cruna {

class StepGraphs {
 public:
  struct Entry {
    int kind;
    const void *p[3];
    int seen = 0;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;  // library launches one replay stands for
  };
  static constexpr size_t kMaxEntries = 64;  // keys beyond these run eagerly
  std::vector<Entry> entries;
  bool off = false;

  ~StepGraphs() {
    for (auto &e : entries)
      if (e.exec) cudaGraphExecDestroy(e.exec);  // freed when its last launch completes
  }
  Entry *find(int kind, const void *a, const void *b, const void *d) {
    for (auto &e : entries)
      if (e.kind == kind && e.p[0] == a && e.p[1] == b && e.p[2] == d) return &e;
    if (entries.size() >= kMaxEntries) return nullptr;
    entries.push_back(Entry{kind, {a, b, d}});
    return &entries.back();
  }
};

GraphScope::GraphScope(cruna_ctx *c) : c_(c) {
  // kernel timing records events between launches and a halo exchange calls back into the host:
  // both need eager steps; so does the legacy default stream, which cannot be captured
  if (c->graphs || !c->graphs_enabled || c->prof_on || c->halo_fn || !c->stream) return;
  own_ = new StepGraphs();
  c->graphs = own_;
}

GraphScope::~GraphScope() {
  if (!own_) return;
  c_->graphs = nullptr;
  delete own_;
}

void graph_step(cruna_ctx *c, int kind, const void *a, const void *b, const void *d,
                const std::function<void()> &body) {
  StepGraphs *G = c->graphs;
  StepGraphs::Entry *e = (G && !G->off) ? G->find(kind, a, b, d) : nullptr;
  if (!e) {
    body();
    return;
  }
  if (e->exec) {
    CRUNA_CUDA_CHECK(cudaGraphLaunch(e->exec, c->stream));
    c->launches += e->launches;
    c->graph_replays++;
    return;
  }
  if (e->seen++ == 0) {
    body();
    return;
  }
  const int64_t l0 = c->launches;
  CRUNA_CUDA_CHECK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  bool ok = true;
  try {
    body();
  } catch (...) {
    ok = false;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t err = cudaStreamEndCapture(c->stream, &graph);
  cudaGraphExec_t exec = nullptr;
  if (ok && err == cudaSuccess && graph) err = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (!ok || err != cudaSuccess || !exec) {
    // the runtime refused the capture (or the step raised): nothing of it ran; clear the non-sticky
    // error, stop recording for this call and run the step eagerly (which raises again if it must)
    cudaGetLastError();
    c->launches = l0;
    G->off = true;
    body();
    return;
  }
  e->exec = exec;
  e->launches = c->launches - l0;
  c->graph_captures++;
  CRUNA_CUDA_CHECK(cudaGraphLaunch(exec, c->stream));
}

}  // namespace cruna

extern "C" {

int cruna_set_graphs(cruna_ctx *c, int on) {
  if (!c) return CRUNA_ERR_ARG;
  c->graphs_enabled = on != 0;
  return CRUNA_OK;
}

int cruna_graph_stats(cruna_ctx *c, int64_t *captured, int64_t *replayed) {
  if (!c) return CRUNA_ERR_ARG;
  if (captured) *captured = c->graph_captures;
  if (replayed) *replayed = c->graph_replays;
  return CRUNA_OK;
}

}  // extern "C"
