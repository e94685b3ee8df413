// solver.cu -- CSR SpMV and the PCG solvers for the reduced SPD system.
//
// The reference solves with a dense partial-pivot LU
// (crates/tpt-fem-sparse/src/lib.rs:244-278), infeasible beyond a few thousand
// dofs; the device path replaces it with preconditioned CG.
//
// One engine serves every method: PCG with reliable updates.  The Krylov
// iteration runs in a working precision T (FP64 for the plain method, FP32
// for mixed precision) on a working copy of the matrix; the solution is
// accumulated in FP64 and, whenever the recursive residual has dropped by
// `delta` since the last update (and always before declaring convergence),
// the true residual r = b - A x is recomputed with the FP64 matrix and
// replaces the recursive one.  The search direction is kept across updates, so
// no Krylov information is lost (a restart would be).  The stopping test is
// always on the TRUE FP64 residual ||b - A x||_2 / ||b||_2.
//
// Kernel structure per iteration (captured in a CUDA graph, BATCH iterations
// per launch; the host reads the state once per batch):
//   K1 spmv_dot : q = A p, pq = p.q
//   K2 update   : alpha = rz/pq; x += alpha p; r -= alpha q; rr = r.r
//                 (Jacobi: also rz' = r.(D^-1 r))
//   [FSAI: t = G r; z = G^T t, rz' = r.z]
//   K3 direction: beta = rz'/rz; p = z + beta p
// Every dot product is reduced deterministically: per-block partials, summed
// in a fixed order by the last block to finish (atomic ticket).  Results are
// bitwise reproducible for a fixed launch configuration.  No kernel waits on
// another kernel or block.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>

#include <type_traits>

#include "lfsai.hpp"
#include "nbsell.cuh"
#include "objects.hpp"
#include "solver_kernels.cuh"

namespace tptfem {

namespace {

// Node-block kernels: blocks per SM in the grid.  Far more than can be
// resident (registers allow ~5): queued blocks start as others finish, which
// balances the uneven per-chunk work better than a grid-stride loop over a
// resident-sized grid (measured on B200: operator 0.242 -> 0.222 ms at
// 4.2M dofs).
constexpr int NB_BLOCKS_PER_SM = 32;

int pick_lanes(int64_t nrows, int64_t nnz) {
  double avg = nrows ? (double)nnz / (double)nrows : 1.0;
  if (avg <= 3) return 2;
  if (avg <= 12) return 4;
  if (avg <= 40) return 8;
  if (avg <= 96) return 16;
  return 32;
}

template <typename TV, typename TX, typename TY, bool DOT>
void launch_spmv(int lanes, int grid, cudaStream_t s, int n, const int* rp, const int* ci, const TV* va, const TX* x,
                 TY* y, PcgState* st, double* partials, bool skip_done) {
  switch (lanes) {
    case 2: spmv_kernel<TV, TX, TY, 2, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials, skip_done); break;
    case 4: spmv_kernel<TV, TX, TY, 4, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials, skip_done); break;
    case 8: spmv_kernel<TV, TX, TY, 8, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials, skip_done); break;
    case 16: spmv_kernel<TV, TX, TY, 16, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials, skip_done); break;
    default: spmv_kernel<TV, TX, TY, 32, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials, skip_done); break;
  }
  TPT_CHECK_LAUNCH();
}

void launch_residual(int lanes, int grid, cudaStream_t s, int n, const int* rp, const int* ci, const double* va,
                     const double* x, const double* b, double* r, double* out2, unsigned* ticket,
                     double* partials) {
  switch (lanes) {
    case 2: residual_f64<2><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    case 4: residual_f64<4><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    case 8: residual_f64<8><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    case 16: residual_f64<16><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    default: residual_f64<32><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
  }
  TPT_CHECK_LAUNCH();
}

}  // namespace

// Default reliable-update trigger of the FP64 Krylov engines: the recursive
// residual drifts little in FP64, so one intermediate replacement (at a drop of
// 1e-6) and the final check suffice; every replacement costs a true residual
// and a preconditioner application.
constexpr double RELIABLE_DELTA_F64 = 1e-6;

// Working-precision PCG engine with reliable updates.
template <typename T>
struct Engine {
  int n = 0;
  int lanes = 8, spmv_grid = 0, vec_grid = 0, batch = 32;
  const int* rp = nullptr;
  const int* ci = nullptr;
  const T* va = nullptr;
  Precond<T> pc;
  DevBuf<T> xl, r, p, q, z, t, dinv;
  DevBuf<double> partials;
  DevBuf<PcgState> st;
  cudaGraphExec_t exec = nullptr;
  // the graph of the other coarse setting (on / off), parked so that solves
  // alternating between the two settings do not capture again
  cudaGraphExec_t exec_alt = nullptr;
  const SystemData* alt_csys = nullptr;
  int alt_cgen = -1;
  void drop_graphs() {
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    if (exec_alt) { cudaGraphExecDestroy(exec_alt); exec_alt = nullptr; }
  }
  // node-block sliced-ELL operator / FSAI factor (FP64 engines only)
  const NbSell* nb = nullptr;
  bool nb_op = false, nb_pc = false, nb_sym = false;
  int nb_grid = 1;
  // aggregation coarse correction (node-block FSAI engines only)
  const SystemData* csys = nullptr;
  int cgen = -1;  // coarse-space generation the pointers in cargs belong to
  CoarseArgs cargs;
  // side stream: the coarse restriction and solve run beside the FSAI lower pass
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  ~Engine() {
    if (exec) cudaGraphExecDestroy(exec);
    if (exec_alt) cudaGraphExecDestroy(exec_alt);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
  }

  void ensure_side() {
    if (side) return;
    int lo = 0, hi = 0;
    TPT_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    TPT_CUDA(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, hi));
    TPT_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    TPT_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  }

  void use_nb(const NbSell* N, bool op, bool pcnb) {
    nb = N;
    nb_op = op;
    nb_pc = pcnb;
    nb_grid = std::max(1, std::min(sm_count() * NB_BLOCKS_PER_SM, ceil_div((int64_t)N->nchunks * 32, SPMV_THREADS)));
    if (partials.n < 2 * (size_t)nb_grid + 2) partials.alloc(2 * (size_t)nb_grid + 2, partials.s);
    drop_graphs();
  }

  // q = A p with the pq reduction (K1).
  void op_dot(cudaStream_t s, const T* x, T* y) {
    if constexpr (std::is_same<T, double>::value) {
      if (nb_op && nb_sym) {
        const NbSell& N = *nb;
#define TPT_NB_SYM(D)                                                                                           \
  nb_spmv_sym<D, true><<<nb_grid, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.ks_lval.p,          \
                                                        N.ks_diag.p, N.u_cptr.p, N.u_col.p, N.ku_base.p, x, y,  \
                                                        st.p, partials.p, true);
        if (N.dpn == 3) { TPT_NB_SYM(3) }
        else if (N.dpn == 2) { TPT_NB_SYM(2) }
        else { TPT_NB_SYM(1) }
#undef TPT_NB_SYM
        TPT_CHECK_LAUNCH();
        return;
      }
      if (nb_op) {
        const NbSell& N = *nb;
        if (N.dpn == 3) nb_spmv<3, true><<<nb_grid, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x, y, st.p, partials.p, true);
        else if (N.dpn == 2) nb_spmv<2, true><<<nb_grid, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x, y, st.p, partials.p, true);
        else nb_spmv<1, true><<<nb_grid, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x, y, st.p, partials.p, true);
        TPT_CHECK_LAUNCH();
        return;
      }
    }
    launch_spmv<T, T, T, true>(lanes, spmv_grid, s, n, rp, ci, va, x, y, st.p, partials.p, true);
  }

  void setup(int n_, const int* rp_, const int* ci_, const T* va_, int64_t nnz, cudaStream_t s, int batch_) {
    n = n_;
    rp = rp_; ci = ci_; va = va_;
    lanes = pick_lanes(n, nnz);
    const int sms = sm_count();
    int per_sm = 0;
    TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_kernel<T, T, T, 8, true>, SPMV_THREADS, 0));
    spmv_grid = std::max(1, std::min(sms * std::max(per_sm, 1), ceil_div((int64_t)n * lanes, SPMV_THREADS)));
    vec_grid = std::max(1, std::min(sms * 8, ceil_div(n, 2 * VEC_THREADS)));
    batch = batch_;
    xl.alloc(n, s); r.alloc(n, s); p.alloc(n, s); q.alloc(n, s); dinv.alloc(n, s);
    partials.alloc(2 * (size_t)std::max(spmv_grid, vec_grid) + 2, s);
    st.alloc(1, s);
    st.zero();
    pc.dinv = dinv.p;
  }

  void ensure_fsai_vectors(cudaStream_t s) {
    if (!z.p) { z.alloc(n, s); t.alloc(n, s); }
  }

  // z = M r with the FSAI factor, rz into st->rz[par ^ 1].
  void apply_fsai(cudaStream_t s, int par) {
    if constexpr (std::is_same<T, double>::value) {
      if (nb_pc) {
        const NbSell& N = *nb;
        if (csys) {  // fork: P^T r and A_c^-1 on the side stream, concurrent with t = G r
          ensure_side();
          TPT_CUDA(cudaEventRecord(ev_fork, s));
          TPT_CUDA(cudaStreamWaitEvent(side, ev_fork, 0));
          coarse_restrict_solve(*csys, r.p, side, &st.p->done);
          TPT_CUDA(cudaEventRecord(ev_join, side));
        }
#define TPT_NB_FSAI(D)                                                                                           \
  nb_fsai_lower<D><<<nb_grid, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.l_pack.p, N.l_tail.p,     \
                                                    N.l_diag.p, pc.sigma2, r.p, t.p, st.p);                       \
  TPT_CHECK_LAUNCH();                                                                                            \
  if (csys) TPT_CUDA(cudaStreamWaitEvent(s, ev_join, 0));                                                        \
  nb_fsai_upper_rz<D><<<nb_grid, SPMV_THREADS, 0, s>>>(N.ngroups, N.u_cptr.p, N.u_col.p, N.u_pack.p, N.u_tail.p,  \
                                                       N.l_diag.p, t.p, r.p, z.p, st.p, partials.p, par, cargs);  \
  TPT_CHECK_LAUNCH();
        if (N.dpn == 3) { TPT_NB_FSAI(3) }
        else if (N.dpn == 2) { TPT_NB_FSAI(2) }
        else { TPT_NB_FSAI(1) }
#undef TPT_NB_FSAI
        return;
      }
    }
    fsai_apply(pc, n, r.p, t.p, z.p, st.p, partials.p, par, s);
  }

  void capture(cudaStream_t s) {
    if (exec) return;
    cudaGraph_t g;
    TPT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < batch; ++it) {
      const int par = it & 1;
      op_dot(s, p.p, q.p);
      if (pc.kind == PC_JACOBI) {
        pcg_update<T, true><<<vec_grid, VEC_THREADS, 0, s>>>(n, par, xl.p, r.p, p.p, q.p, dinv.p, st.p, partials.p);
        TPT_CHECK_LAUNCH();
        pcg_direction<T, true><<<vec_grid, VEC_THREADS, 0, s>>>(n, par, r.p, p.p, dinv.p, nullptr, st.p);
      } else {
        pcg_update<T, false><<<vec_grid, VEC_THREADS, 0, s>>>(n, par, xl.p, r.p, p.p, q.p, nullptr, st.p, partials.p);
        TPT_CHECK_LAUNCH();
        apply_fsai(s, par);
        pcg_direction<T, false><<<vec_grid, VEC_THREADS, 0, s>>>(n, par, r.p, p.p, nullptr, z.p, st.p);
      }
      TPT_CHECK_LAUNCH();
    }
    TPT_CUDA(cudaStreamEndCapture(s, &g));
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    TPT_CUDA(e);
  }

  // r = (T) r_hi; xl = 0; z = M r, rz -> rz[0]; p = z + (rz / rz_old) p; done = 0.
  void reset(const double* r_hi, double upd2, cudaStream_t s) {
    reset_residual<T><<<vec_grid, VEC_THREADS, 0, s>>>(n, r_hi, r.p, xl.p, pc.kind == PC_JACOBI ? dinv.p : nullptr,
                                                       st.p, partials.p, upd2);
    TPT_CHECK_LAUNCH();
    if (pc.kind != PC_JACOBI) apply_fsai(s, 1);  // parity 1 writes rz[0]
    reset_direction<T><<<vec_grid, VEC_THREADS, 0, s>>>(n, r.p, p.p, pc.kind == PC_JACOBI ? dinv.p : nullptr,
                                                        pc.kind == PC_JACOBI ? nullptr : z.p, st.p);
    TPT_CHECK_LAUNCH();
  }
};

struct SolverWork {
  Engine<double> f64;      // Jacobi, FP64 (node-block operator when the system allows it)
  Engine<double> f64_csr;  // Jacobi, FP64, CSR operator only (TPTFEM_SOLVE_CSR_ONLY)
  Engine<float> f32;       // Jacobi, FP32 Krylov
  Engine<double> f64_fsai; // FSAI (FP16 factor), FP64 Krylov
  Engine<double> f64_lf;   // learned FSAI (FP16 factor), FP64 Krylov
  FsaiFactor fsai, lf;
  LfGraph lgraph;
  const FsaiFactor* nb_factor = nullptr;  // factor whose blocks S.nb holds
  bool f64_ready = false, f64_csr_ready = false, f32_ready = false, fsai_ready = false, fsai_failed = false;
  bool lf_ready = false, lf_engine = false;
  int seen_gen[8] = {-1, -1, -1, -1, -1, -1, -1, -1};  // per method: value generation last set up for
  DevBuf<double> rhi;   // FP64 true residual
  DevBuf<double> sc;    // scalars
  DevBuf<unsigned> tk;  // tickets for standalone reductions
  DevBuf<double> partials;
  PcgState* h_state = nullptr;
  ~SolverWork() {
    if (h_state) cudaFreeHost(h_state);
  }
};

SystemData::~SystemData() = default;

namespace {

// The coarse set-up beside the network forward (TPTFEM_COARSE_OVERLAP=0: after it).
bool coarse_overlap() {
  static const bool on = [] {
    const char* e = std::getenv("TPTFEM_COARSE_OVERLAP");
    return !(e && e[0] == '0');
  }();
  return on;
}

void ensure_work(SystemData& S) {
  cudaStream_t s = S.ctx->stream;
  if (!S.work) {
    S.work = std::make_shared<SolverWork>();
    TPT_CUDA(cudaMallocHost(&S.work->h_state, sizeof(PcgState)));
    S.work->rhi.alloc(std::max<int64_t>(S.n_free, 1), s);
    S.work->sc.alloc(8, s);
    S.work->tk.alloc(8, s);
    S.work->tk.zero();
    S.work->partials.alloc(4096, s);
  }
}

// Node-block engines use the symmetric half storage of K unless the caller
// asks for the full operator (TPTFEM_SOLVE_FULL_OPERATOR); switching drops the
// engine's captured graph.
// Operator storage for this solve (symmetric half or full); on a fresh set-up
// its values are taken from the CSR again unless they were filled since the
// previous solve's set-up.
void select_nb_mode(SystemData& S, Engine<double>& E, const tptfem_solver_opts& o) {
  if (!E.nb_op) return;
  const bool sym = !(o.flags & TPTFEM_SOLVE_FULL_OPERATOR);
  if (sym) nb_build_sym(S);
  if (!sym && S.nb.full_stale) nb_refill_values(S, false);
  else if ((o.flags & TPTFEM_SOLVE_FRESH_SETUP) && !S.nb.fresh_fill) nb_refill_values(S, sym);
  S.nb.fresh_fill = false;
  if (E.nb_sym != sym) {
    E.nb_sym = sym;
    E.drop_graphs();
  }
}

// Coarse correction for an FSAI engine (TPTFEM_SOLVE_COARSE): geometry once
// per system, A_c and its inverse whenever the preconditioner is set up
// afresh.  Returns the coarse size in use (0: off).
int select_coarse(SystemData& S, Engine<double>& E, const tptfem_solver_opts& o, bool fresh) {
  bool want = (o.flags & TPTFEM_SOLVE_COARSE) && E.nb_pc;
  PhaseTimer timer(S.ctx->stream, "coarse space");
  // default: about one aggregate per 2000 node groups for vector problems (6 or
  // 3 rigid modes each) and per 700 for scalar ones (one constant mode each),
  // between 8 and 3000.  Measured (fresh set-up + solve, learned FSAI): at
  // 280x70x70, 700 aggregates (3300 coarse unknowns) 96.9 ms against 98.9 with
  // 500, 105.3 with 350 and 103.5 with 1000, where the dense coarse set-up
  // grows faster than the iterations fall; at 400x100x100, 1000-1365
  // aggregates 287-291 ms against 309 with 700; for the 128^3 Poisson
  // random-field problems 2744 (23.9 ms per solve against 26.1 ms with 729).
  const int aggs = o.coarse_aggregates > 0 ? o.coarse_aggregates : coarse_default_aggregates(S);
  if (want) want = coarse_build(S, aggs);
  if (want && (fresh || !S.coarse.ready)) want = coarse_assemble(S);
  if (want && !S.coarse.ready) want = false;
  const SystemData* target = want ? &S : nullptr;
  if (E.csys != target || (want && E.cgen != S.coarse.generation)) {
    // park the current graph; take the parked one if it was captured for the
    // new setting (and, with the coarse space, for the same coarse geometry)
    cudaGraphExec_t parked = E.exec;
    const SystemData* parked_csys = E.csys;
    const int parked_cgen = E.cgen;
    E.exec = nullptr;
    if (E.exec_alt && E.alt_csys == target && (!want || E.alt_cgen == S.coarse.generation)) {
      E.exec = E.exec_alt;
      E.exec_alt = nullptr;
    }
    if (E.exec_alt) cudaGraphExecDestroy(E.exec_alt);
    E.exec_alt = parked;
    E.alt_csys = parked_csys;
    E.alt_cgen = parked_cgen;
    E.csys = target;
    E.cgen = S.coarse.generation;
    E.cargs = CoarseArgs{};
    if (want) {
      E.cargs.agg = S.coarse.agg.p;
      E.cargs.y = S.coarse.y.p;
      E.cargs.cm = S.coarse.cm.p;
    }
  }
  return want ? S.coarse.nc : 0;
}

void flag_check(tptfem_context* ctx, const char* msg) {
  TPT_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  TPT_REQUIRE(ctx->h_pinned[0] == 0, TPTFEM_ERR_NUMERIC, msg);
}

template <typename T>
void prepare_jacobi(SystemData& S, Engine<T>& E, const T* va, int batch) {
  cudaStream_t s = S.ctx->stream;
  E.setup((int)S.n_free, S.row_ptr.p, S.col.p, va, S.nnz, s, batch);
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  jacobi_diag<T><<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, E.dinv.p,
                                                         S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  flag_check(S.ctx, "reduced matrix has a missing or non-positive diagonal entry (not SPD)");
  E.pc.kind = PC_JACOBI;
}

template <typename T>
void refresh_jacobi(SystemData& S, Engine<T>& E) {
  cudaStream_t s = S.ctx->stream;
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  jacobi_diag<T><<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, E.dinv.p,
                                                         S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  flag_check(S.ctx, "reduced matrix has a missing or non-positive diagonal entry (not SPD)");
}

// ||b - A x||^2 in FP64 into W.rhi / returned.
double true_residual2(SystemData& S, const double* x) {
  SolverWork& W = *S.work;
  cudaStream_t s = S.ctx->stream;
  int lanes = pick_lanes(S.n_free, S.nnz);
  int grid = std::max(1, std::min(sm_count() * 8, ceil_div(S.n_free * lanes, SPMV_THREADS)));
  launch_residual(lanes, grid, s, (int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, x, S.fred.p, W.rhi.p, W.sc.p + 1,
                  W.tk.p + 1, W.partials.p);
  double h;
  TPT_CUDA(cudaMemcpyAsync(&h, W.sc.p + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  return h;
}

double norm2_b(SystemData& S) {
  SolverWork& W = *S.work;
  cudaStream_t s = S.ctx->stream;
  int grid = std::max(1, std::min(sm_count() * 4, ceil_div(S.n_free, VEC_THREADS)));
  sumsq_kernel<<<grid, VEC_THREADS, 0, s>>>((int)S.n_free, S.fred.p, W.sc.p, W.tk.p, W.partials.p);
  TPT_CHECK_LAUNCH();
  double h;
  TPT_CUDA(cudaMemcpyAsync(&h, W.sc.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  return h;
}

// PCG with reliable updates; see the file comment.  Returns iterations.
template <typename T>
int64_t run_reliable(SystemData& S, Engine<T>& E, double tol, double delta, int64_t max_it, double bnorm,
                     tptfem_solve_stats& st) {
  SolverWork& W = *S.work;
  cudaStream_t s = S.ctx->stream;
  const double target2 = tol * tol * bnorm * bnorm;
  const double final2 = 0.25 * target2;  // recursive test a little below the true one
  E.capture(s);
  // start: x = 0, r = b
  S.x.zero();
  E.p.zero();
  double rr = true_residual2(S, S.x.p);
  if (rr <= target2) return 0;
  // p = z + beta*p with rz_old = +inf gives p = z on the first reset
  init_state<<<1, 1, 0, s>>>(E.st.p, (int)std::min<int64_t>(max_it, 1 << 30));
  TPT_CHECK_LAUNCH();
  E.reset(W.rhi.p, std::max(delta * delta * rr, final2), s);
  int64_t iters = 0;
  for (;;) {
    TPT_CUDA(cudaMemcpyAsync(W.h_state, E.st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    TPT_CUDA(cudaStreamSynchronize(s));
    const PcgState h = *W.h_state;
    if (h.done == 0) {
      TPT_CUDA(cudaGraphLaunch(E.exec, s));
      continue;
    }
    iters = h.iters;
    if (h.done == 2) {
      st.iterations = iters;
      TPT_REQUIRE(false, TPTFEM_ERR_BREAKDOWN, "PCG breakdown: p.Ap <= 0 or NaN (matrix not SPD?)");
    }
    // reliable update: accumulate x in FP64 and replace r by the true residual
    accumulate<T><<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, E.xl.p, S.x.p);
    TPT_CHECK_LAUNCH();
    rr = true_residual2(S, S.x.p);
    st.outer_steps += 1;
    if (debug_trace())
      fprintf(stderr, "[tptfem] update %d: iters=%d done=%d recursive=%.3e true=%.3e target=%.3e\n",
              st.outer_steps, h.iters, h.done, std::sqrt(h.rr) / bnorm, std::sqrt(rr) / bnorm, tol);
    if (rr <= target2) break;
    if (h.done == 3 || iters >= max_it) break;
    E.reset(W.rhi.p, std::max(delta * delta * rr, final2), s);
  }
  return iters;
}

}  // namespace

namespace {

void ensure_val32(SystemData& S) {
  cudaStream_t s = S.ctx->stream;
  if (!S.val32.p) {
    S.val32.alloc(S.nnz, s);
    to_f32<<<ceil_div(S.nnz, 256), 256, 0, s>>>(S.nnz, S.val.p, S.val32.p);
    TPT_CHECK_LAUNCH();
  }
}

// FP64 Krylov engine preconditioned by an FSAI factor whose values are set.
void prepare_fsai_engine(SystemData& S, Engine<double>& E, const FsaiFactor& F, int batch) {
  cudaStream_t s = S.ctx->stream;
  E.setup((int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, S.nnz, s, batch);
  E.ensure_fsai_vectors(s);
  E.pc.kind = PC_FSAI;
  E.pc.n = (int)F.n;
  E.pc.lanes = pick_lanes(F.n, F.nnz);
  E.pc.grid = std::max(1, std::min(sm_count() * 8, ceil_div(F.n * E.pc.lanes, SPMV_THREADS)));
  E.pc.sigma2 = F.sigma2.p;
  E.pc.g_rp = F.rp.p; E.pc.g_ci = F.ci.p; E.pc.g_va = F.va.p;
}

// The row-wise CSR apply (no node-block factor) needs the explicit transpose.
void ensure_csr_fsai(SystemData& S, Engine<double>& E, FsaiFactor& F) {
  if (E.nb_pc) return;
  fsai_build_transpose(S, F);
  if (E.pc.gt_va != F.tva.p) {
    E.pc.gt_rp = F.trp.p; E.pc.gt_ci = F.tci.p; E.pc.gt_va = F.tva.p;
    E.drop_graphs();
  }
}

// Learned factor values: network forward on this system, converted to the
// FP64 factor of A and installed (sigma^2 FP32, L FP16).  False if invalid.
bool learned_factor(SystemData& S, SolverWork& W) {
  cudaStream_t s = S.ctx->stream;
  {
    PhaseTimer t(S.ctx->stream, "factor pattern");
    // the network inputs build the node-block operator anyway; with it the
    // factor pattern comes from its group adjacency
    if (S.dpn <= 3) nb_build_operator(S);
    fsai_build_pattern(S, W.lf);
  }
  if (W.lf.overflow) return false;
  if (!W.lgraph.ready) {
    PhaseTimer t(S.ctx->stream, "network inputs");
    W.lgraph.prepare(S, W.lf);
  }
  {
    PhaseTimer t(S.ctx->stream, "network forward + Kaporin");
    if (!lf_forward(S, W.lf, W.lgraph, S.lmodel->prm.p)) return false;
  }
  PhaseTimer t(S.ctx->stream, "factor conversion");
  DevBuf<double> sig2, lva;
  sig2.alloc(W.lf.n, s);
  lva.alloc(std::max<int64_t>(W.lf.nnz, 1), s);
  lf_factor_fp64(S, W.lf, W.lgraph, sig2.p, lva.p);
  return fsai_set_values(S, W.lf, sig2.p, lva.p);
}

}  // namespace

LfGraph& system_lf_graph(SystemData& S, FsaiFactor** F) {
  ensure_work(S);
  SolverWork& W = *S.work;
  fsai_build_pattern(S, W.lf);
  TPT_REQUIRE(!W.lf.overflow, TPTFEM_ERR_CREATION, "factor pattern rows exceed the device limit");
  if (!W.lgraph.ready) W.lgraph.prepare(S, W.lf);
  *F = &W.lf;
  return W.lgraph;
}

void system_solve(SystemData& S, const tptfem_solver_opts& o_in, tptfem_solve_stats& st) {
  tptfem_context* ctx = S.ctx;
  tptfem_solver_opts o = o_in;
  cudaStream_t s = ctx->stream;
  const double tol = o.rel_tol > 0 ? o.rel_tol : 1e-10;
  const int64_t max_it = o.max_iter > 0 ? o.max_iter : 100000;
  int batch = o.batch > 0 ? o.batch : 32;
  batch += batch & 1;
  st = tptfem_solve_stats{};
  TPT_REQUIRE(o.solver >= TPTFEM_SOLVER_JACOBI_PCG && o.solver <= TPTFEM_SOLVER_LEARNED_FSAI_PCG,
              TPTFEM_ERR_INVALID_ARG, "unknown solver");
  int solver = o.solver;
  if (S.n_free == 0) {
    st.solver_used = solver;
    return;
  }
  ensure_work(S);
  SolverWork& W = *S.work;
  {  // values changed by tptfem_system_refresh since this method last set up: set up afresh
    const int slot = solver + ((o.flags & TPTFEM_SOLVE_CSR_ONLY) ? 4 : 0);
    if (W.seen_gen[slot] != S.value_gen) {
      if (W.seen_gen[slot] >= 0) o.flags |= TPTFEM_SOLVE_FRESH_SETUP;
      W.seen_gen[slot] = S.value_gen;
    }
  }
  if (solver == TPTFEM_SOLVER_LEARNED_FSAI_PCG) {
    TPT_REQUIRE(S.lmodel != nullptr, TPTFEM_ERR_INVALID_ARG, "no learned model attached to this system");
    TPT_CUDA(cudaEventRecord(ctx->ev[0], s));
    const bool fresh = (o.flags & TPTFEM_SOLVE_FRESH_SETUP) || !W.lf_ready;
    if (o.flags & TPTFEM_SOLVE_FRESH_SETUP) W.lgraph.ready = false;  // A^ and node features from the values again
    // Every fresh set-up after the first (engine, node-block layout and coarse
    // geometry in place): the coarse matrix and its inverse are formed on the
    // engine's side stream while the network computes the factor on this one;
    // both only read the operator values.
    bool coarse_pending = false;
    if (fresh && W.lf_engine && W.f64_lf.nb_pc && (o.flags & TPTFEM_SOLVE_COARSE) && coarse_overlap() &&
        S.coarse.state == 1 &&
        S.coarse.target == (o.coarse_aggregates > 0 ? o.coarse_aggregates : coarse_default_aggregates(S))) {
      Engine<double>& E = W.f64_lf;
      {
        PhaseTimer t(S.ctx->stream, "symmetric operator");
        select_nb_mode(S, E, o);
      }
      E.ensure_side();
      TPT_CUDA(cudaEventRecord(E.ev_fork, s));
      TPT_CUDA(cudaStreamWaitEvent(E.side, E.ev_fork, 0));
      coarse_pending = coarse_assemble_async(S, E.side);
      TPT_CUDA(cudaEventRecord(E.ev_join, E.side));
    }
    bool ok = !fresh || learned_factor(S, W);
    if (coarse_pending) {  // the inverse is needed from here on; a failed Cholesky leaves the coarse space off
      TPT_CUDA(cudaStreamWaitEvent(s, W.f64_lf.ev_join, 0));
      coarse_finish(S, s);
    }
    if (fresh && ok && !W.lf_engine) {
      prepare_fsai_engine(S, W.f64_lf, W.lf, batch);
      PhaseTimer t(S.ctx->stream, "engine + node-block layout");
      if (!(o.flags & TPTFEM_SOLVE_CSR_ONLY) && nb_build_operator(S)) {
        const bool nbpc = nb_fill_factor(S, W.lf);
        W.f64_lf.use_nb(&S.nb, true, nbpc);
        if (nbpc) W.nb_factor = &W.lf;
      }
      W.lf_engine = true;
    } else if (fresh && ok && W.f64_lf.nb_pc) {
      nb_fill_factor(S, W.lf);
      W.nb_factor = &W.lf;
    }
    W.lf_ready = ok;
    if (ok) {
      if (W.f64_lf.nb_pc && W.nb_factor != &W.lf) {
        nb_fill_factor(S, W.lf);
        W.nb_factor = &W.lf;
      }
      st.solver_used = solver;
      if (!coarse_pending) {
        PhaseTimer t(S.ctx->stream, "symmetric operator");
        select_nb_mode(S, W.f64_lf, o);
      }
      st.coarse_size = select_coarse(S, W.f64_lf, o, fresh && !coarse_pending);
      TPT_CUDA(cudaEventRecord(ctx->ev[1], s));
      const double bb = norm2_b(S);
      const double bnorm = std::sqrt(bb);
      int64_t iters = 0;
      bool broke = false;
      if (bb == 0.0) {
        S.x.zero();
      } else {
        const double delta = o.inner_rel_tol > 0 ? o.inner_rel_tol : RELIABLE_DELTA_F64;
        try {
          ensure_csr_fsai(S, W.f64_lf, W.lf);
          iters = run_reliable<double>(S, W.f64_lf, tol, delta, max_it, bnorm, st);
        } catch (const Error& e) {
          if (e.status != TPTFEM_ERR_BREAKDOWN) throw;
          broke = true;
        }
      }
      const double rel = bb == 0.0 ? 0.0 : std::sqrt(true_residual2(S, S.x.p)) / bnorm;
      if (!broke && rel <= tol) {
        TPT_CUDA(cudaEventRecord(ctx->ev[2], s));
        TPT_CUDA(cudaEventSynchronize(ctx->ev[2]));
        float ms0 = 0.f, ms1 = 0.f;
        TPT_CUDA(cudaEventElapsedTime(&ms0, ctx->ev[0], ctx->ev[1]));
        TPT_CUDA(cudaEventElapsedTime(&ms1, ctx->ev[1], ctx->ev[2]));
        st.iterations = iters;
        st.rel_residual = rel;
        st.setup_ms = ms0;
        st.solve_ms = ms1;
        return;
      }
    }
    // the learned factor was invalid, broke down or did not converge: the plain
    // FP64 Jacobi-PCG solves the system instead
    tptfem_solver_opts fb = o;
    fb.solver = TPTFEM_SOLVER_JACOBI_PCG;
    system_solve(S, fb, st);
    st.fell_back = 1;
    return;
  }
  TPT_CUDA(cudaEventRecord(ctx->ev[0], s));
  if (solver == TPTFEM_SOLVER_FSAI_MP_PCG && W.fsai_ready && W.f64_fsai.nb_pc && W.nb_factor != &W.fsai &&
      !(o.flags & TPTFEM_SOLVE_FRESH_SETUP)) {
    nb_fill_factor(S, W.fsai);
    W.nb_factor = &W.fsai;
  }
  if (o.flags & TPTFEM_SOLVE_FRESH_SETUP) {
    // keep patterns, graphs and buffers; recompute every value of the preconditioner
    if (solver == TPTFEM_SOLVER_FSAI_MP_PCG && W.fsai_ready) {
      if (!fsai_classic(S, W.fsai)) {
        W.fsai_ready = false;
        W.fsai_failed = true;
      } else if (W.f64_fsai.nb_pc) {
        nb_fill_factor(S, W.fsai);
        W.nb_factor = &W.fsai;
      }
    } else if (solver == TPTFEM_SOLVER_JACOBI_PCG && (o.flags & TPTFEM_SOLVE_CSR_ONLY) && W.f64_csr_ready) {
      refresh_jacobi<double>(S, W.f64_csr);
    } else if (solver == TPTFEM_SOLVER_JACOBI_PCG && !(o.flags & TPTFEM_SOLVE_CSR_ONLY) && W.f64_ready) {
      refresh_jacobi<double>(S, W.f64);
    } else if (solver == TPTFEM_SOLVER_MP_PCG && W.f32_ready) {
      refresh_jacobi<float>(S, W.f32);
    }
  }
  if (solver == TPTFEM_SOLVER_FSAI_MP_PCG) {
    if (!W.fsai_ready && !W.fsai_failed) {
      if (fsai_classic(S, W.fsai)) {
        prepare_fsai_engine(S, W.f64_fsai, W.fsai, batch);
        if (!(o.flags & TPTFEM_SOLVE_CSR_ONLY) && nb_build_operator(S)) {
          const bool nbpc = nb_fill_factor(S, W.fsai);
          W.f64_fsai.use_nb(&S.nb, true, nbpc);
          if (nbpc) W.nb_factor = &W.fsai;
        }
        W.fsai_ready = true;
      } else {
        W.fsai_failed = true;
      }
    }
    if (!W.fsai_ready) {  // factor not SPD or rows too long: the plain method takes over
      solver = TPTFEM_SOLVER_JACOBI_PCG;
      st.fell_back = 1;
    }
  }
  const bool csr_only = (o.flags & TPTFEM_SOLVE_CSR_ONLY) != 0;
  if (solver == TPTFEM_SOLVER_JACOBI_PCG && csr_only && !W.f64_csr_ready) {
    prepare_jacobi<double>(S, W.f64_csr, S.val.p, batch);
    W.f64_csr_ready = true;
  }
  if (solver == TPTFEM_SOLVER_JACOBI_PCG && !csr_only && !W.f64_ready) {
    prepare_jacobi<double>(S, W.f64, S.val.p, batch);
    if (nb_build_operator(S)) W.f64.use_nb(&S.nb, true, false);
    W.f64_ready = true;
  }
  if (solver == TPTFEM_SOLVER_MP_PCG && !W.f32_ready) {
    ensure_val32(S);
    prepare_jacobi<float>(S, W.f32, S.val32.p, batch);
    W.f32_ready = true;
  }
  st.solver_used = solver;
  if (solver == TPTFEM_SOLVER_FSAI_MP_PCG) {
    select_nb_mode(S, W.f64_fsai, o);
    st.coarse_size = select_coarse(S, W.f64_fsai, o, (o.flags & TPTFEM_SOLVE_FRESH_SETUP) != 0);
  }
  TPT_CUDA(cudaEventRecord(ctx->ev[1], s));
  const double bb = norm2_b(S);
  const double bnorm = std::sqrt(bb);
  int64_t iters = 0;
  if (bb == 0.0) {
    S.x.zero();
  } else if (solver == TPTFEM_SOLVER_JACOBI_PCG) {
    const double delta = o.inner_rel_tol > 0 ? o.inner_rel_tol : RELIABLE_DELTA_F64;
    Engine<double>& EJ = csr_only ? W.f64_csr : W.f64;
    select_nb_mode(S, EJ, o);
    iters = run_reliable<double>(S, EJ, tol, delta, max_it, bnorm, st);
  } else if (solver == TPTFEM_SOLVER_MP_PCG) {
    const double delta = o.inner_rel_tol > 0 ? o.inner_rel_tol : 0.05;
    iters = run_reliable<float>(S, W.f32, tol, delta, max_it, bnorm, st);
  } else {
    const double delta = o.inner_rel_tol > 0 ? o.inner_rel_tol : RELIABLE_DELTA_F64;
    ensure_csr_fsai(S, W.f64_fsai, W.fsai);
    iters = run_reliable<double>(S, W.f64_fsai, tol, delta, max_it, bnorm, st);
  }
  const double rel = bb == 0.0 ? 0.0 : std::sqrt(true_residual2(S, S.x.p)) / bnorm;
  TPT_CUDA(cudaEventRecord(ctx->ev[2], s));
  TPT_CUDA(cudaEventSynchronize(ctx->ev[2]));
  float ms0 = 0.f, ms1 = 0.f;
  TPT_CUDA(cudaEventElapsedTime(&ms0, ctx->ev[0], ctx->ev[1]));
  TPT_CUDA(cudaEventElapsedTime(&ms1, ctx->ev[1], ctx->ev[2]));
  st.iterations = iters;
  st.rel_residual = rel;
  st.setup_ms = ms0;
  st.solve_ms = ms1;
  TPT_REQUIRE(rel <= tol, TPTFEM_ERR_NOT_CONVERGED, "PCG did not reach the requested residual");
}

int64_t system_fsai_classic(SystemData& S) {
  ensure_work(S);
  SolverWork& W = *S.work;
  if (!W.fsai_ready && !W.fsai_failed) {
    if (fsai_classic(S, W.fsai)) {
      prepare_fsai_engine(S, W.f64_fsai, W.fsai, 32);
      W.fsai_ready = true;
    } else {
      W.fsai_failed = true;
    }
  }
  return W.fsai_ready ? W.fsai.nnz : -1;
}

const FsaiFactor* system_block_factor(SystemData& S, bool learned) {
  ensure_work(S);
  SolverWork& W = *S.work;
  FsaiFactor& F = learned ? W.lf : W.fsai;
  if (learned) {
    TPT_REQUIRE(S.lmodel, TPTFEM_ERR_INVALID_ARG, "no network attached to the system");
    if (S.dpn <= 3) nb_build_operator(S);  // the pattern from the group adjacency, as in a solve
  }
  fsai_build_pattern(S, F);
  if (F.overflow) return nullptr;
  fsai_build_transpose(S, F);  // before the values, which then fill the transpose too
  const bool ok = learned ? learned_factor(S, W) : fsai_classic(S, F);
  return ok ? &F : nullptr;
}

namespace {
__global__ void half_to_f64(int64_t n, const __half* __restrict__ a, double* __restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)__half2float(a[i]);
}
__global__ void f32_to_f64(int64_t n, const float* __restrict__ a, double* __restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}
}  // namespace

void system_fsai_download(const SystemData& S, int64_t* rp, int64_t* ci, double* lva, double* sig2) {
  TPT_REQUIRE(S.work && S.work->fsai_ready, TPTFEM_ERR_INVALID_ARG, "no FSAI factor on this system");
  const FsaiFactor& F = S.work->fsai;
  cudaStream_t s = S.ctx->stream;
  std::vector<int> hrp(F.n + 1), hci(F.nnz);
  F.rp.download(hrp.data(), hrp.size());
  F.ci.download(hci.data(), hci.size());
  DevBuf<double> tmp;
  tmp.alloc(std::max<int64_t>(std::max<int64_t>(F.nnz, F.n), 1), s);
  if (lva && F.nnz) {
    half_to_f64<<<ceil_div(F.nnz, 256), 256, 0, s>>>(F.nnz, F.va.p, tmp.p);
    TPT_CHECK_LAUNCH();
    tmp.download(lva, F.nnz);
  }
  TPT_CUDA(cudaStreamSynchronize(s));
  if (sig2) {
    f32_to_f64<<<ceil_div(F.n, 256), 256, 0, s>>>(F.n, F.sigma2.p, tmp.p);
    TPT_CHECK_LAUNCH();
    tmp.download(sig2, F.n);
  }
  TPT_CUDA(cudaStreamSynchronize(s));
  if (rp)
    for (size_t i = 0; i < hrp.size(); ++i) rp[i] = hrp[i];
  if (ci)
    for (size_t i = 0; i < hci.size(); ++i) ci[i] = hci[i];
}

// Average device time of the solver's SpMV kernels on this system (diagnostic
// for the roofline report): FP64 and FP32 CSR, `reps` back-to-back launches
// each, timed with events on the context stream.
void system_profile_spmv(SystemData& S, int reps, double* ms_f64, double* ms_f32, double* ms_nb, double* nb_bytes,
                         double* ms_nbs, double* nbs_bytes) {
  cudaStream_t s = S.ctx->stream;
  ensure_work(S);
  ensure_val32(S);
  DevBuf<double> x64, y64;
  DevBuf<float> x32, y32;
  x64.alloc(S.n_free, s); y64.alloc(S.n_free, s); x32.alloc(S.n_free, s); y32.alloc(S.n_free, s);
  x64.zero(); x32.zero();
  const int lanes = pick_lanes(S.n_free, S.nnz);
  int per_sm = 0;
  TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_kernel<double, double, double, 8, true>,
                                                         SPMV_THREADS, 0));
  const int grid = std::max(1, std::min(sm_count() * std::max(per_sm, 1), ceil_div(S.n_free * lanes, SPMV_THREADS)));
  auto timeit = [&](auto launch) {
    launch();
    TPT_CUDA(cudaEventRecord(S.ctx->ev[0], s));
    for (int i = 0; i < reps; ++i) launch();
    TPT_CUDA(cudaEventRecord(S.ctx->ev[1], s));
    TPT_CUDA(cudaEventSynchronize(S.ctx->ev[1]));
    float ms = 0.f;
    TPT_CUDA(cudaEventElapsedTime(&ms, S.ctx->ev[0], S.ctx->ev[1]));
    return (double)ms / reps;
  };
  *ms_f64 = timeit([&] {
    launch_spmv<double, double, double, false>(lanes, grid, s, (int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, x64.p,
                                               y64.p, nullptr, nullptr, false);
  });
  *ms_f32 = timeit([&] {
    launch_spmv<float, float, float, false>(lanes, grid, s, (int)S.n_free, S.row_ptr.p, S.col.p, S.val32.p, x32.p,
                                            y32.p, nullptr, nullptr, false);
  });
  *ms_nb = -1.0;
  if (nb_build_operator(S)) {
    if (S.nb.full_stale) nb_refill_values(S, false);
    const NbSell& N = S.nb;
    const int g = std::max(1, std::min(sm_count() * NB_BLOCKS_PER_SM, ceil_div((int64_t)N.nchunks * 32, SPMV_THREADS)));
    *ms_nb = timeit([&] {
      if (N.dpn == 3) nb_spmv<3, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x64.p, y64.p, nullptr, nullptr, false);
      else if (N.dpn == 2) nb_spmv<2, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x64.p, y64.p, nullptr, nullptr, false);
      else nb_spmv<1, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x64.p, y64.p, nullptr, nullptr, false);
      TPT_CHECK_LAUNCH();
    });
    *nb_bytes = (double)N.k_slots * 32 * (4 + 8 * N.dpn * N.dpn) + (double)(N.nchunks + 1) * 4 +
                16.0 * (double)S.n_free;
    nb_build_sym(S);
    *ms_nbs = timeit([&] {
#define TPT_NB_SYM(D)                                                                                             \
  nb_spmv_sym<D, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.ks_lval.p, N.ks_diag.p,     \
                                                   N.u_cptr.p, N.u_col.p, N.ku_base.p, x64.p, y64.p, nullptr,      \
                                                   nullptr, false);
      if (N.dpn == 3) { TPT_NB_SYM(3) }
      else if (N.dpn == 2) { TPT_NB_SYM(2) }
      else { TPT_NB_SYM(1) }
#undef TPT_NB_SYM
      TPT_CHECK_LAUNCH();
    });
    // bytes the half storage must move: lower and diagonal blocks, lower
    // columns, upper columns and block indices, chunk pointers, x and y
    const double d2 = (double)(N.dpn * N.dpn);
    *nbs_bytes = (double)N.l_slots * 32 * (4 + 8 * d2) + (double)N.nchunks * 32 * 8 * d2 +
                 (double)N.u_slots * 32 * 8 + 2.0 * (N.nchunks + 1) * 4 + 16.0 * (double)S.n_free;
  }
}

void system_values_changed(SystemData& S) {
  ++S.value_gen;
  if (S.val32.p) {  // the FP32 copy used by the mixed-precision engine is refreshed in place
    to_f32<<<ceil_div(S.nnz, 256), 256, 0, S.ctx->stream>>>(S.nnz, S.val.p, S.val32.p);
    TPT_CHECK_LAUNCH();
  }
  if (S.work) S.work->lgraph.ready = false;  // network inputs derive from the values
  S.coarse.ready = false;
  nb_refresh_values(S);
}

void nb_operator_apply(SystemData& S, const double* x, double* y) {
  if (!S.nb.sym_built && S.nb.full_stale) nb_refill_values(S, false);
  const NbSell& N = S.nb;
  cudaStream_t s = S.ctx->stream;
  const int g = std::max(1, std::min(sm_count() * NB_BLOCKS_PER_SM, ceil_div((int64_t)N.nchunks * 32, SPMV_THREADS)));
  if (N.sym_built) {
#define TPT_NB_SYM(D)                                                                                             \
  nb_spmv_sym<D, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.ks_lval.p, N.ks_diag.p,     \
                                                   N.u_cptr.p, N.u_col.p, N.ku_base.p, x, y, nullptr, nullptr, false);
    if (N.dpn == 3) { TPT_NB_SYM(3) }
    else if (N.dpn == 2) { TPT_NB_SYM(2) }
    else { TPT_NB_SYM(1) }
#undef TPT_NB_SYM
  } else {
    if (N.dpn == 3) nb_spmv<3, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x, y, nullptr, nullptr, false);
    else if (N.dpn == 2) nb_spmv<2, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x, y, nullptr, nullptr, false);
    else nb_spmv<1, false><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.k_cptr.p, N.k_col.p, N.k_val.p, x, y, nullptr, nullptr, false);
  }
  TPT_CHECK_LAUNCH();
}

void nb_operator_apply_modes(SystemData& S, const double* X, double* Y, const unsigned char* gcol, int colour,
                             const unsigned* cmask, cudaStream_t s) {
  nb_build_sym(S);
  const NbSell& N = S.nb;
  const int g = std::max(1, std::min(sm_count() * NB_BLOCKS_PER_SM, ceil_div((int64_t)N.nchunks * 32, SPMV_THREADS)));
  if (N.dpn == 3)
    nb_spmv_sym_multi<3, 6><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.ks_lval.p, N.ks_diag.p,
                                                       N.u_cptr.p, N.u_col.p, N.ku_base.p, X, Y, gcol, colour, cmask);
  else if (N.dpn == 2)
    nb_spmv_sym_multi<2, 3><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.ks_lval.p, N.ks_diag.p,
                                                       N.u_cptr.p, N.u_col.p, N.ku_base.p, X, Y, gcol, colour, cmask);
  else
    nb_spmv_sym_multi<1, 1><<<g, SPMV_THREADS, 0, s>>>(N.ngroups, N.l_cptr.p, N.l_col.p, N.ks_lval.p, N.ks_diag.p,
                                                       N.u_cptr.p, N.u_col.p, N.ku_base.p, X, Y, gcol, colour, cmask);
  TPT_CHECK_LAUNCH();
}

void csr_matvec_f64(tptfem_context* ctx, int64_t nrows, const int* rp, const int* ci, const double* va,
                    const double* x, double* y) {
  if (nrows == 0) return;
  int lanes = 4;
  int grid = std::max(1, std::min(sm_count() * 8, ceil_div(nrows * lanes, SPMV_THREADS)));
  launch_spmv<double, double, double, false>(lanes, grid, ctx->stream, (int)nrows, rp, ci, va, x, y, nullptr, nullptr,
                                             false);
}

}  // namespace tptfem
