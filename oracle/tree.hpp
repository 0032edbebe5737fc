// CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Restatement of FMM2DTree<K> from vaishna77/RCS
// include/AIFMMTree2D_3D_memory_optimized.hpp (3-D build, USE_THREE), active
// paths only: tree build and lists (:52-331, :425-476, :576-668), skeletons
// (:681-760, :917-1077, :1155-1284), leaf/non-leaf P2P (:3343-3504), the
// elimination (:3537-4509, :4599-4747), the recompressions that the
// elimination calls (:1573-1656, :2116-2306, :2454-2596, :2878-2959,
// :3159-3340) and the solve sweeps (:3506-3535, :4749-4907).  The
// std::map<int,Mat> members are kept as std::map with operator[] at the same
// places as the reference, because the reference iterates some of them and
// auto-inserted empty entries change those iterations.
#pragma once
#include <map>
#include <utility>
#include <vector>

#include "lowrank.hpp"

namespace orc {

struct SolverInputs {
  double xmin, xmax, ymin, ymax, zmin, zmax;
  int leafSize, tol_pow, nLevelsInput, fillin_rank, fillin_tol;
  std::vector<V3> locations;
};

struct Box {
  double maxPivot_L2P = 0.0, maxPivot_P2M = 0.0;
  bool ILActive = true;
  int boxNumber = -1, parentNumber = -1;
  std::vector<int> interactionList, neighborList;
  bool Eliminated = false;
  int NumMultipoles = 0, NumLocals = 0;
  V3 center;
  Mat particles, multipoles, locals, particle_rhs, multipole_rhs, local_rhs;
  std::map<int, Mat> M2L, P2P, M2P, P2L, L2P_f, P2M_f, M2M_f;
  Mat L2M_f, L2P, P2M;
  std::vector<int> chargeLocations;
  std::vector<int> incoming_chargePoints, incoming_checkPoints, outgoing_chargePoints, outgoing_checkPoints;
  Mat Ac, Ar;
};

struct TreeStats {
  double tAssemble = 0, tFactor = 0, tSolve = 0;
  long nRRQR = 0, nCompressP2P = 0, nCompressP2L = 0;
};

class Tree {
 public:
  const Kernel* K;
  bool realMode;
  int nLevels, N, startLevel = 0;
  double L, eta;
  int TOL_POW, fill_in_TOL_POW;
  double fillInTolerance;
  int nChild = 8;
  std::vector<int> nBoxesPerLevel;
  std::vector<double> boxSideLength;
  std::vector<std::vector<Box>> tree;
  std::vector<V3> particles;
  std::vector<std::pair<int, int>> P2L_M2P, P2Pq;
  int fillin_rankVec[64];
  double domain[6];
  TreeStats stats;

  Tree(const SolverInputs& in, const Kernel* K, bool realMode);
  // AIFMM constructor sequence (AIFMM.cpp:7-93)
  void build();
  void factorize();                           // eliminate_phase_efficient
  void solve(const Mat& rhs, Mat& x);         // backSubstitute1..3 + getPhi
  int getAvgLeafSize() const;
  int getAvgMultipoles() const;
  double findMemory();
  double findMemoryAfterFactorize();
  int maxRank() const;

  // pieces
  void createTree();
  void assign_Center_Location();
  void assign_Tree_Interactions();
  bool admissibility(int j, int child, int other);
  void assignChargeLocations();
  void assignNonLeafChargeLocations();
  void getNodes();
  void getNodes_incoming_box(int j, int k);
  void getNodes_outgoing_box(int j, int k);
  void get_L2P_P2M_box(int j, int k);
  void assemble_M2L();
  void free_charge_and_checkPoints();
  void initialise_phase();
  void initialise_P2P_Leaf_Level();
  void initialise_P2P_NonLeafLevel(int j);
  void deleteM2L(int j);

  // elimination
  bool is_well_separated(int j, int k, int l);
  void eliminate_x(int j, int k);
  void eliminate_z(int j, int k);
  void compress_P2P_myRRQR(int j, int k, int b, const Mat& old_L2P, const Mat& old_P2M, const Mat& P2PToBeCompressed,
                           Mat& new_L2P, Mat& new_P2M_transpose, Mat& Rk, Mat& Rn, Mat& Rn_prime, Mat& newM2L);
  void compress_P2P_Two_Ways_myRRQR(int j, int k, int b);
  void compress_M2P_myRRQR(int j, int k, int b, Mat& new_L2P, Mat& M2L);
  void compress_P2L_myRRQR(int j, int k, int b, Mat& new_P2M_transpose, Mat& M2L);
  void compress_M2P_P2L_myRRQR(int j, int k, int b);
  void update_other_M2Ls_at_k_old(int j, int k, int b, const Mat& new_L2P);
  void update_other_M2Ls_at_b_old(int j, int k, int b, const Mat& new_P2M_transpose);
  void update_parent_L2P_old(int j, int k, const Mat& new_L2P);
  void update_parent_P2M_old(int j, int b, const Mat& new_P2M_transpose);

  // solve
  void assign_Leaf_rhs(const Mat& charges);
  void assign_particle_rhs_NonLeafLevel(int j);
  void rhs_eliminate_x(int j, int k);
  void rhs_eliminate_z(int j, int k);
  void rhs_eliminate_phase_efficient();
  void solve_particles_at_base_level(int j);
  void back_substitution_phase();
  void getx(Mat& x);
  void reorder(Mat& x);
};

}  // namespace orc
