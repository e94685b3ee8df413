// lfsai.hpp -- learned FSAI network (lfsai.cu): sizes, per-system buffers and
// the forward / backward / optimiser entry points used by the C ABI.
#pragma once
#include "objects.hpp"

namespace tptfem {

constexpr int LF_D0 = 8;      // input node features
constexpr int LF_H = 16;      // hidden width
constexpr int LF_LAYERS = 2;  // message-passing layers

// Per-system network buffers (matrix-derived inputs and activations).
struct LfGraph {
  bool ready = false;
  int n = 0;
  int64_t nnz = 0, nnzl = 0;
  DevBuf<float> ahat;   // A^ values (CSR of the reduced matrix)
  DevBuf<double> dis;   // d^-1/2
  DevBuf<float> x0;     // node features (n x LF_D0)
  DevBuf<float> al;     // A^ at the factor pattern entries
  DevBuf<float> ya[LF_LAYERS], yb[LF_LAYERS], h[LF_LAYERS];
  DevBuf<float> P, Q, sig, lhat;
  DevBuf<int> flag;     // lf_kaporin: bit 0 row too long, bit 1 q <= 0
  // node-block form (all dofs of every free node free): A^ as dpn x dpn blocks
  // on the node-group adjacency of the node-block operator, row-major per block
  bool nb = false;
  int nb_checked = -1;  // -1 not checked, 0 no, 1 yes (the pattern is fixed per system)
  DevBuf<float> ablk;
  void prepare(SystemData& S, const FsaiFactor& F);
};

struct LfModel {
  tptfem_context* ctx = nullptr;
  DevBuf<float> prm, grad, m1, m2;
  int step = 0;
};

int lf_param_count();
void lf_init_params(uint64_t seed, float* host);
// Forward to L^ and sig; false if a row was too long or q_i <= 0.
bool lf_forward(const SystemData& S, const FsaiFactor& F, LfGraph& G, const float* prm);
// Kaporin loss (1/n) sum_i log q_i; when grad != nullptr adds d loss / d params to grad.
double lf_loss_grad(const SystemData& S, const FsaiFactor& F, LfGraph& G, const float* prm, float* grad);
void lf_adam_step(cudaStream_t s, int np, float* prm, const float* grad, float* m1, float* m2, int step, float lr,
                  float clip);
void lf_factor_fp64(const SystemData& S, const FsaiFactor& F, const LfGraph& G, double* sig2, double* lva);

// solver.cu: per-system learned factor (pattern, graph buffers) for training / solves.
LfGraph& system_lf_graph(SystemData& S, FsaiFactor** F);

}  // namespace tptfem

struct tptfem_lfsai {
  std::shared_ptr<tptfem::LfModel> d;
};
