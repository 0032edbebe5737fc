// GPU AIFMM solver: the FMM2DTree<K> of vaishna77/RCS
// (include/AIFMMTree2D_3D_memory_optimized.hpp) with every block in HBM.
// Host code keeps the tree topology, the per-box maps of block handles and the
// fill-in queues -- the same control flow as the reference, so the plain FP64
// path takes the same pivots, ranks and elimination order -- and issues all
// arithmetic as kernels on the context stream.
#pragma once
#include <map>
#include <memory>
#include <utility>
#include <vector>

#include "dmat.cuh"
#include "lowrank.cuh"
#include "mlp.cuh"

namespace aifmm {

struct SolverParams {
  int leafSize = 64, tol_pow = 8, nLevelsInput = 0, fillin_rank = 0, fillin_tol = 10;
  int realMode = 0;      // electrostatics: real Householder sign in RRQR
  size_t aca_budget = (size_t)24 << 30;  // bytes of ACA workspace per launch
  bool phaseTiming = false;              // synchronise at phase boundaries for exact phase times
  bool orthoShortcut = true;             // skip partition 1 of RRQR for orthonormal old bases
  int precision = 0;                     // 1: elimination GEMMs in split TF32 on the tensor cores
  int drop_pow = 0;                      // fill-in queue threshold 10^-drop_pow (0: 10^-tol_pow; <0: drop all)
};

struct SolverStats {
  double t_assemble = 0, t_factor = 0, t_solve = 0;
  double t_rrqr = 0, t_compress = 0, t_elim_x = 0, t_elim_z = 0, t_nonleaf = 0;
  double t_lu = 0, t_msolve = 0, t_schur = 0;  // inside eliminate_x/z: box LU, multi-column solves, Schur GEMMs
  double flops_factor = 0;  // complex-counted algorithmic flops issued by the factorization
  long nRRQR = 0, nRRQRShort = 0, nCompressP2P = 0, nCompressP2L = 0, nACA = 0, nACARetry = 0;
  long kernels = 0;
  long nSolveGraph = 0, nSolveCapture = 0;  // solves replayed from a captured graph / graphs captured
  double t_aca = 0;          // host time of the ACA phase (launches, retries, read-backs)
  double aca_ws_bytes = 0;   // ACA workspace bytes allocated over all launches (retries included)
  long nACALaunches = 0;     // ACA launches (chunks of problems that fit the workspace budget)
};

// One ACA problem of the build: its features, the workspace rank bound it was
// first launched with, and the rank the adaptive ACA found.
struct ACARecord {
  RankFeatures x;
  int rmax0, rank;
};

// A captured CUDA graph of the whole solve sweep for one right-hand-side
// count: it reads `in` and writes `out`, buffers of the plan, and every
// intermediate block it touches stays reserved by `hold` while it exists.
// The graph's kernels read the factorization's blocks at their addresses, so
// a plan is dropped whenever they change (factorize, rewind, load).
struct SolvePlan {
  aifmm_ctx* ctx = nullptr;
  int nrhs = 0;
  DMat in, out;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::shared_ptr<CaptureHold> hold;
  long launches = 0;  // kernels per replay
  ~SolvePlan();
};

struct DBox {
  double maxPivot_L2P = 0.0, maxPivot_P2M = 0.0;
  bool ILActive = true;
  std::vector<int> IL, NB;
  bool Eliminated = false;
  int NumMultipoles = 0, NumLocals = 0;
  double center[3] = {0, 0, 0};
  DMat particles, multipoles, locals, particle_rhs, multipole_rhs, local_rhs;
  std::map<int, DMat> M2L, P2P, M2P, P2L, L2P_f, P2M_f, M2M_f;
  DMat L2M_f, L2P, P2M;
  std::vector<int> chargeLocations, in_charge, in_check, out_charge, out_check;
  DMat Ac, Ar;
  DLU luP2P, luL2M;  // factors of P2P[k] and L2M_f, alive during the box's elimination
  // P2P[k]^{-1} and -L2M_f^{-1}, kept for the solve sweeps (the reference
  // refactorizes the blocks there); applied as multi-SM products
  DMat invP2P, negInvL2M;
  // L2P has orthonormal columns / P2M orthonormal rows because a recompression
  // of this box produced them (not the ACA interpolation, not a parent update)
  bool l2pOrtho = false, p2mOrtho = false;
  bool hasLuP2P = false, hasLuL2M = false;
};

class Solver {
 public:
  aifmm_kernel* K;
  aifmm_ctx* ctx;
  Ops ops;
  SolverParams prm;
  SolverStats stats;
  int N = 0, nLevels = 0, startLevel = 0;
  double L = 0, eta = 0, fillInTolerance = 0;
  int nChild = 8;
  std::vector<int> nBoxesPerLevel;
  std::vector<double> boxSideLength;
  std::vector<std::vector<DBox>> tree;
  std::vector<double> particles;  // N x 3
  std::vector<std::pair<int, int>> P2L_M2P, P2Pq;
  int fillin_rankVec[64];
  double domain[6];
  bool factored = false;
  std::vector<ACARecord> acaLog;  // every ACA problem of the build, in launch order

  // xyz (N x 3) and dom (xmin, xmax, ymin, ymax, zmin, zmax) replace the
  // kernel's unknown locations and their bounding box when given, as
  // inputsToSolverClass::locations and xmin..zmax do in the reference.
  Solver(aifmm_kernel* k, const SolverParams& p, const double* xyz = nullptr, const double* dom = nullptr);
  void build();
  void factorize();
  // rhs: N x nrhs (device), returns x: N x nrhs (device).  With graphSolve
  // (the default) the first solve for a right-hand-side count after a
  // factorization captures the sweep as a CUDA graph and every solve,
  // that one included, replays it: one graph launch instead of thousands of
  // kernel launches issued from the host.
  DMat solve(const DMat& rhs);
  bool graphSolve = true;
  void dropPlan() { plan_.reset(); }  // the next solve captures again

  int avgLeafSize() const;
  int avgMultipoles() const;
  int maxRank() const;
  double memoryGB(bool afterFactor);
  // Keep a device copy of the assembled (unfactorized) state / restore it so
  // that factorize() can run again on the same operator.
  void checkpoint();
  void rewind();
  // Write the factorized state to a file / replace this solver's state by a
  // file's (the kernel must have the file's unknown count); a loaded solver
  // solves without assembling or factorizing.
  void save(const std::string& path);
  void load(const std::string& path);

 private:
  void createTree();
  void assignCenters();
  void assignInteractions();
  void assignCharges();
  void getNodesLevel(int j);
  void runACA(int j, bool incoming);
  RankFeatures rankFeatures(int j, int k, int nr, int nc) const;
  void getL2PP2MBox(int j, int k);
  void assembleM2L();
  void initP2PLeaf();
  void initP2PNonLeaf(int j);
  void deleteM2L(int j);
  bool wellSeparated(int j, int k, int l) const;
  void eliminateX(int j, int k);
  void eliminateZ(int j, int k);
  void compressP2PTwoWays(int j, int k, int b);
  // newM2L of compressP2P_myRRQR from the new bases (the products after its two RRQRs)
  void compressP2PM2L(int j, int k, int b, const DMat& oldL2P, const DMat& oldP2M, const DMat& nL2P,
                      const DMat& nP2Mt, const DMat& Rkp, DMat& newM2L, bool prefixL, bool prefixM);
  void compressM2PP2L(int j, int k, int b);
  // prefix: the new basis starts with the old one (the RRQR kept an
  // orthonormal old basis), so the basis change is a partial identity and
  // the products below reduce to row / column selection with zero padding.
  void updateOtherM2LsAtK(int j, int k, int b, const DMat& nL2P, bool prefix);
  void updateOtherM2LsAtB(int j, int k, int b, const DMat& nP2Mt, bool prefix);
  void updateParentL2P(int j, int k, const DMat& nL2P, bool prefix);
  void updateParentP2M(int j, int b, const DMat& nP2Mt, bool prefix);
  // old blocks -> rows x old.c (first rows kept, zero below) / old.r x cols
  // (first columns kept, zero right); one grouped copy for all of them
  void resizeRows(const std::vector<DMat*>& blocks, int rows);
  void resizeCols(const std::vector<DMat*>& blocks, int cols);
  // One recompression RRQR: A = [old basis (partition columns) | fill-in].
  struct RRQRJob {
    DMat A;
    int partition = 0;
    double inputPivot = 0;
    int fillRank = 0;
    bool orthoPanel = false;  // the old basis has orthonormal columns
    DMat Q;                   // out: Q_trunc
    double maxPivot = 0;      // out
    bool prefix = false;      // out: Q starts with the old basis
  };
  void rrqrBatch(const std::vector<RRQRJob*>& jobs);  // independent jobs, one launch
  DMat solveSweeps(const DMat& rhs);  // the sweep, enqueued without synchronising
  void capturePlan(int nrhs);
  std::unique_ptr<SolvePlan> plan_;
  void assignLeafRhs(const DMat& rhs);
  void rhsEliminateX(int j, int k);
  void rhsEliminateZ(int j, int k);
  void baseSolve(int j);
  void factorBase(int j);
  void backSubstitute();
  void gatherBlocks(const std::vector<std::vector<int>*>& rows, const std::vector<std::vector<int>*>& cols,
                    std::vector<DMat*>& outs);
  std::vector<std::vector<DBox>> deepCopy(std::vector<std::vector<DBox>>& src);
  void treeOrder();
  int nrhs_ = 1;
  bool leafPermReady_ = false;
  std::shared_ptr<DevBuf> leafPerm_;  // tree-order position -> unknown id
  std::vector<int> leafOff_;          // leaf box -> first tree-order position
  std::vector<std::vector<DBox>> saved_;
  bool hasSaved_ = false;
  DLU baseLU_;             // factors of the base-level system (factorBase)
  bool baseReady_ = false;
};

}  // namespace aifmm

struct aifmm_solver {
  std::unique_ptr<aifmm::Solver> s;
};
