// Batched FMM evaluations captured in one CUDA graph.
#pragma once
#include <memory>

#include "laplace.cuh"

namespace b2 {

// Per-problem device pointers (arrays of n entries; a null array means the
// argument is absent for every problem).
struct BatchIO {
  const double* const* charge = nullptr;
  const double* const* dipstr = nullptr;
  const double* const* dipvec = nullptr;
  double* const* pot = nullptr;
  double* const* grad = nullptr;
  double* const* hess = nullptr;
  double* const* pottarg = nullptr;
  double* const* gradtarg = nullptr;
  double* const* hesstarg = nullptr;
};

struct BatchGraph;

// Evaluates every plan once (ordinary launches, synchronised: checks the
// arguments), then captures one evaluation of each plan into a graph whose
// `nbranch` branches run concurrently.  The plans and pointers must outlive
// the graph.
int batch_graph_create(int n, LapPlan* const* plans, const BatchIO& io, int nbranch,
                       BatchGraph** out);
int batch_graph_launch(BatchGraph* g, cudaStream_t st);
int batch_graph_status(BatchGraph* g);  // IER_TIMEOUT if a tensor-core wait gave up
size_t batch_graph_nodes(const BatchGraph* g);
void batch_graph_free(BatchGraph* g);

}  // namespace b2
