// Many independent FMM evaluations in one CUDA graph.
//
// Each problem is a plan (tree, lists, sorted points, buffers: laplace.cu).
// The graph holds one evaluation of every plan, spread over `nbranch`
// independent branches (fork/join through events on a capturing stream), so
// small problems that cannot fill the GPU on their own run side by side and
// a whole batch costs one graph launch instead of hundreds of kernel
// launches per problem.  The mixed near fields of all plans (one density
// chunk each) run as one persistent pass over the work items of every tree
// (p2p_batch_launch, one launch per group of density count, output level
// and density kind) between the plans' far fields and their unsorts:
//     fork -> plans up to the far field -> join -> batched near field ->
//     fork -> the plans' unsorts -> join.
#include "batch.cuh"

#include "lap_mixed.cuh"

#include <algorithm>
#include <vector>

namespace b2 {

struct BatchGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<LapPlan*> plans;
  P2PBatch* near = nullptr;  // the batched near-field pass (null: none deferred)
  size_t nodes = 0;
  ~BatchGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (near) p2p_batch_free(near);
  }
};

int batch_graph_create(int n, LapPlan* const* plans, const BatchIO& io, int nbranch,
                       BatchGraph** out) {
  *out = nullptr;
  if (n < 1 || nbranch < 1 || !plans) return IER_BADARG;
  nbranch = std::min(nbranch, n);
  std::unique_ptr<BatchGraph> G(new BatchGraph());
  cudaStream_t s0 = nullptr;
  std::vector<cudaStream_t> br(nbranch, nullptr);
  std::vector<cudaEvent_t> join(nbranch, nullptr);
  cudaEvent_t fork = nullptr;
  auto cleanup = [&]() {
    for (auto& s : br)
      if (s) cudaStreamDestroy(s);
    for (auto& e : join)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (s0) cudaStreamDestroy(s0);
  };
  auto eval = [&](int i, cudaStream_t s, int part) {
    return lap_plan_eval_part(
        plans[i], io.charge ? io.charge[i] : nullptr, io.dipstr ? io.dipstr[i] : nullptr,
        io.dipvec ? io.dipvec[i] : nullptr, io.pot ? io.pot[i] : nullptr,
        io.grad ? io.grad[i] : nullptr, io.hess ? io.hess[i] : nullptr,
        io.pottarg ? io.pottarg[i] : nullptr, io.gradtarg ? io.gradtarg[i] : nullptr,
        io.hesstarg ? io.hesstarg[i] : nullptr, s, false, nullptr, part);
  };
  std::vector<char> defer(n, 0);
  std::vector<P2PBatchEntry> entries;
  for (int i = 0; i < n; i++)
    if (lap_plan_defers_near(plans[i])) {
      defer[i] = 1;
      lap_plan_near_entries(plans[i], entries);
    }
  try {
    B2_CHECK(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
    for (auto& s : br) B2_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (auto& e : join) B2_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    B2_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    // one ordinary evaluation of every plan first: checks the arguments and
    // performs every one-time set-up (kernel attributes) outside the capture
    for (int i = 0; i < n; i++) {
      int r = eval(i, s0, 0);
      if (r != IER_OK) {
        cleanup();
        return r;
      }
    }
    if (!entries.empty()) {
      // the batched pass once outside the capture too (its kernel attributes;
      // it only adds to the plans' tree-order buffers, which every
      // evaluation rewrites)
      G->near = p2p_batch_create(entries);
      p2p_batch_launch(G->near, s0);
    }
    B2_CHECK(cudaStreamSynchronize(s0));
    for (int i = 0; i < n; i++) {
      int r = lap_plan_status(plans[i]);
      if (r != IER_OK) {
        cleanup();
        return r;
      }
    }
    B2_CHECK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    int rc = IER_OK;
    try {
      auto fork_join = [&](auto body) {
        B2_CHECK(cudaEventRecord(fork, s0));
        for (auto& s : br) B2_CHECK(cudaStreamWaitEvent(s, fork, 0));
        body();
        for (int b = 0; b < nbranch; b++) {
          B2_CHECK(cudaEventRecord(join[b], br[b]));
          B2_CHECK(cudaStreamWaitEvent(s0, join[b], 0));
        }
      };
      fork_join([&] {
        for (int i = 0; i < n && rc == IER_OK; i++) rc = eval(i, br[i % nbranch], defer[i] ? 1 : 0);
      });
      if (G->near && rc == IER_OK) {
        p2p_batch_launch(G->near, s0);
        fork_join([&] {
          for (int i = 0; i < n && rc == IER_OK; i++)
            if (defer[i]) rc = eval(i, br[i % nbranch], 2);
        });
      }
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s0, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    B2_CHECK(cudaStreamEndCapture(s0, &G->graph));
    if (rc != IER_OK) {
      cleanup();
      return rc;
    }
    B2_CHECK(cudaGraphInstantiate(&G->exec, G->graph, 0));
    B2_CHECK(cudaGraphGetNodes(G->graph, nullptr, &G->nodes));
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
  G->plans.assign(plans, plans + n);
  *out = G.release();
  return IER_OK;
}

int batch_graph_launch(BatchGraph* g, cudaStream_t st) {
  if (!g) return IER_BADARG;
  B2_CHECK(cudaGraphLaunch(g->exec, st));
  return IER_OK;
}

int batch_graph_status(BatchGraph* g) {
  if (!g) return IER_BADARG;
  for (LapPlan* p : g->plans) {
    int r = lap_plan_status(p);
    if (r != IER_OK) return r;
  }
  return IER_OK;
}

size_t batch_graph_nodes(const BatchGraph* g) { return g ? g->nodes : 0; }

void batch_graph_free(BatchGraph* g) { delete g; }

}  // namespace b2
