// CPU oracle -- TEST INFRASTRUCTURE ONLY.  Restatement of FMM2DTree<K>
// (include/AIFMMTree2D_3D_memory_optimized.hpp, cited as T:line below).
#include "tree.hpp"

#include <omp.h>

#include <chrono>

namespace orc {

static double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------ constructor, T:52-165
Tree::Tree(const SolverInputs& in, const Kernel* K_, bool rm) : K(K_), realMode(rm) {
  particles = in.locations;
  TOL_POW = in.tol_pow;
  fill_in_TOL_POW = in.fillin_tol;
  fillInTolerance = std::pow(10, -1.0 * TOL_POW);
  domain[0] = in.xmin; domain[1] = in.xmax;
  domain[2] = in.ymin; domain[3] = in.ymax;
  domain[4] = in.zmin; domain[5] = in.zmax;
  double Lx = in.xmax - in.xmin, Ly = in.ymax - in.ymin, Lz = in.zmax - in.zmin;
  L = std::max({Lx, Ly, Lz});
  N = (int)in.locations.size();
  const int q = N / in.leafSize;  // integer division as in T:132
  if (q <= 0) nLevels = 2;
  else nLevels = std::max(2, int(std::floor(std::log(q) / std::log(8))));
  if (in.nLevelsInput > 0) nLevels = in.nLevelsInput;  // extension: T:62 leaves it unused
  if (nLevels >= 63) fail("too many levels");
  eta = std::sqrt(3) * 2;
  nBoxesPerLevel.push_back(1);
  boxSideLength.push_back(L);
  for (int k = 1; k <= nLevels; ++k) {
    nBoxesPerLevel.push_back(nChild * nBoxesPerLevel[k - 1]);
    boxSideLength.push_back(0.5 * boxSideLength[k - 1]);
  }
  for (int k = 0; k < 64; ++k) fillin_rankVec[k] = 0;
  int temp = 5, i = 0;
  for (int k = nLevels; k >= 2; --k) {  // T:148-156
    fillin_rankVec[k] = temp;
    ++i;
    if (i % 3 == 0) temp += 5;
  }
}

void Tree::createTree() {  // T:167-192
  tree.clear();
  tree.resize(nLevels + 1);
  for (int j = 0; j <= nLevels; ++j) {
    tree[j].resize(nBoxesPerLevel[j]);
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      tree[j][k].boxNumber = k;
      tree[j][k].parentNumber = (j == 0) ? -1 : k / nChild;
    }
  }
}

void Tree::assign_Center_Location() {  // T:425-463
  tree[0][0].center = V3((domain[0] + domain[1]) / 2.0, (domain[2] + domain[3]) / 2.0, (domain[4] + domain[5]) / 2.0);
  static const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  static const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  static const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int j = 0; j < nLevels; ++j) {
    int J = j + 1;
    double shift = 0.5 * boxSideLength[J];
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      const V3 c = tree[j][k].center;
      for (int ch = 0; ch < 8; ++ch) {
        V3& cc = tree[J][8 * k + ch].center;
        cc[0] = sx[ch] < 0 ? c[0] - shift : c[0] + shift;
        cc[1] = sy[ch] < 0 ? c[1] - shift : c[1] + shift;
        cc[2] = sz[ch] < 0 ? c[2] - shift : c[2] + shift;
      }
    }
  }
}

bool Tree::admissibility(int j, int child, int other) {  // T:277-293
  const V3 &a = tree[j][child].center, &b = tree[j][other].center;
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  double d = std::sqrt(dx * dx + dy * dy + dz * dz);
  double etaLocal = eta;
  if (j == nLevels) etaLocal = eta / 2.0;
  if (d > etaLocal * boxSideLength[j] + boxSideLength[nLevels] / 2.0) {
    tree[j][child].interactionList.push_back(other);
    return true;
  }
  tree[j][child].neighborList.push_back(other);
  return false;
}

void Tree::assign_Tree_Interactions() {  // T:266-331
  tree[0][0].neighborList.push_back(0);
  for (int j = 0; j < nLevels; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      for (int c = 0; c < nChild; ++c) {
        int child = nChild * k + c;
        for (size_t n = 0; n < tree[j][k].neighborList.size(); ++n) {
          int nn = tree[j][k].neighborList[n];
          for (int cc = 0; cc < nChild; ++cc) admissibility(j + 1, child, nn * nChild + cc);
        }
      }
  int flag = -1;
  for (int j = 0; j <= nLevels; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      if (flag != 0 && tree[j][k].interactionList.size() != 0) {
        startLevel = j;
        flag = 0;
      }
}

void Tree::assignChargeLocations() {  // T:576-625
  for (int i = 0; i < N; ++i) tree[0][0].chargeLocations.push_back(i);
  for (int j = 0; j < nLevels; ++j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      int J = j + 1, Kp = 8 * k;
      const V3 c = tree[j][k].center;
      for (int index : tree[j][k].chargeLocations) {
        const V3& p = particles[index];
        int ch;
        if (p[2] <= c[2]) {
          if (p[0] <= c[0]) ch = (p[1] <= c[1]) ? 0 : 3;
          else ch = (p[1] <= c[1]) ? 1 : 2;
        } else {
          if (p[0] <= c[0]) ch = (p[1] <= c[1]) ? 4 : 7;
          else ch = (p[1] <= c[1]) ? 5 : 6;
        }
        tree[J][Kp + ch].chargeLocations.push_back(index);
      }
    }
}

void Tree::assignNonLeafChargeLocations() {  // T:659-668
  for (int j = nLevels - 1; j >= 0; j--)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      auto& cl = tree[j][k].chargeLocations;
      cl.clear();
      for (int i = 0; i < nChild; ++i) {
        auto& c = tree[j + 1][nChild * k + i].chargeLocations;
        cl.insert(cl.end(), c.begin(), c.end());
      }
    }
}

// ------------------------------------------------------------ skeletons
static void truncateTo(std::vector<int>& v, size_t n) {
  if (v.size() > n) v.resize(n);
}

void Tree::getNodes_outgoing_box(int j, int k) {  // T:994-1077
  std::vector<int> boxA;
  if (j == nLevels) boxA = tree[j][k].chargeLocations;
  else
    for (int c = 0; c < nChild; ++c) {
      auto& v = tree[j + 1][nChild * k + c].outgoing_chargePoints;
      boxA.insert(boxA.end(), v.begin(), v.end());
    }
  std::vector<int> IL;
  for (int kIL : tree[j][k].interactionList) {
    if (j == nLevels) {
      auto& v = tree[j][kIL].chargeLocations;
      IL.insert(IL.end(), v.begin(), v.end());
    } else {
      for (int c = 0; c < nChild; ++c) {
        auto& v = tree[j + 1][nChild * kIL + c].incoming_checkPoints;
        IL.insert(IL.end(), v.begin(), v.end());
      }
    }
  }
  const int n_rows = (int)IL.size(), n_cols = (int)boxA.size();
  if (n_cols > 0 && n_rows > 0) {
    ACAResult r;
    acaOnlyNodes2(*K, std::pow(10, -TOL_POW), IL, boxA, r);
    tree[j][k].Ar = r.Ar;
    if (r.rank > 0) {
      for (int rb : r.rowBases) tree[j][k].outgoing_checkPoints.push_back(IL[rb]);
      for (int cb : r.colBases) tree[j][k].outgoing_chargePoints.push_back(boxA[cb]);
    }
  } else if (n_rows == 0) {
    tree[j][k].ILActive = false;
    tree[j][k].outgoing_chargePoints = boxA;
  }
}

void Tree::getNodes_incoming_box(int j, int k) {  // T:1155-1256
  std::vector<int> boxA;
  if (j == nLevels) boxA = tree[j][k].chargeLocations;
  else
    for (int c = 0; c < nChild; ++c) {
      auto& v = tree[j + 1][nChild * k + c].incoming_checkPoints;
      boxA.insert(boxA.end(), v.begin(), v.end());
    }
  std::vector<int> IL;
  for (int kIL : tree[j][k].interactionList) {
    if (j == nLevels) {
      auto& v = tree[j][kIL].chargeLocations;
      IL.insert(IL.end(), v.begin(), v.end());
    } else {
      for (int c = 0; c < nChild; ++c) {
        auto& v = tree[j + 1][nChild * kIL + c].outgoing_chargePoints;
        IL.insert(IL.end(), v.begin(), v.end());
      }
    }
  }
  const int n_rows = (int)boxA.size(), n_cols = (int)IL.size();
  if (n_rows > 0 && n_cols > 0) {
    ACAResult r;
    acaOnlyNodes2(*K, std::pow(10, -TOL_POW), boxA, IL, r);
    tree[j][k].Ac = r.Ac;
    if (r.rank > 0) {
      for (int rb : r.rowBases) tree[j][k].incoming_checkPoints.push_back(boxA[rb]);
      for (int cb : r.colBases) tree[j][k].incoming_chargePoints.push_back(IL[cb]);
    }
  } else if (n_cols == 0) {
    tree[j][k].ILActive = false;
    tree[j][k].incoming_checkPoints = boxA;
  }
}

void Tree::get_L2P_P2M_box(int j, int k) {  // T:681-732
  Box& B = tree[j][k];
  if (B.incoming_checkPoints.size() < B.outgoing_chargePoints.size()) {
    truncateTo(B.outgoing_checkPoints, B.incoming_checkPoints.size());
    truncateTo(B.outgoing_chargePoints, B.incoming_checkPoints.size());
  } else {
    truncateTo(B.incoming_checkPoints, B.outgoing_chargePoints.size());
    truncateTo(B.incoming_chargePoints, B.outgoing_chargePoints.size());
  }
  const int nin = (int)B.incoming_checkPoints.size();
  const int nout = (int)B.outgoing_checkPoints.size();
  if (B.ILActive) {
    Mat temp1 = B.Ac.block(0, 0, B.Ac.r, nin);
    B.L2P = Mat::Zero(B.Ac.r, nin);
    if (nin > 0) {
      Mat D1 = K->getMatrix(B.incoming_checkPoints, B.incoming_chargePoints);
      LU lu(D1.adjoint());
      B.L2P = lu.solve(temp1.adjoint()).adjoint();
    }
    Mat temp2 = B.Ar.block(0, 0, nout, B.Ar.c);
    B.P2M = Mat(nout, B.Ar.c);
    if (nout > 0) {
      Mat D2 = K->getMatrix(B.outgoing_checkPoints, B.outgoing_chargePoints);
      LU lu(D2);
      B.P2M = lu.solve(temp2);
    }
  } else {
    B.L2P = Mat::Identity(nin, nin);
    const int no = (int)B.outgoing_chargePoints.size();
    B.P2M = Mat::Identity(no, no);
  }
  if (B.Ac.size() > 0) B.maxPivot_L2P = maxColumnNorm(B.Ac.block(0, 0, B.Ac.r, nin));
  if (B.Ar.size() > 0) B.maxPivot_P2M = maxColumnNorm(B.Ar.block(0, 0, nout, B.Ar.c).adjoint());
}

void Tree::getNodes() {  // T:917-944, :755-760
  for (int j = nLevels; j >= startLevel; j--) {
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) getNodes_incoming_box(j, k);
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) getNodes_outgoing_box(j, k);
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) get_L2P_P2M_box(j, k);
  }
}

void Tree::assemble_M2L() {  // T:1258-1273
  for (int j = startLevel; j <= nLevels; j++) {
    // pre-insert keys serially; std::map insertion is not thread-safe
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      for (int kIL : tree[j][k].interactionList) tree[j][k].M2L[kIL];
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k)
      for (int kIL : tree[j][k].interactionList)
        tree[j][k].M2L[kIL] = K->getMatrix(tree[j][k].incoming_checkPoints, tree[j][kIL].outgoing_chargePoints);
  }
}

void Tree::free_charge_and_checkPoints() {  // T:1275-1284
  for (int j = startLevel; j <= nLevels; j++)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      tree[j][k].outgoing_chargePoints.clear();
      tree[j][k].incoming_checkPoints.clear();
      tree[j][k].Ar = Mat(0, 0);
      tree[j][k].Ac = Mat(0, 0);
    }
}

void Tree::initialise_phase() {  // T:3343-3370
  for (int j = startLevel; j <= nLevels; j++)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      tree[j][k].NumMultipoles = tree[j][k].P2M.r;
      tree[j][k].NumLocals = tree[j][k].L2P.c;
    }
  for (int j = startLevel; j <= nLevels; j++)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      tree[j][k].local_rhs = Mat::Zero(tree[j][k].NumMultipoles, 1);
      tree[j][k].multipole_rhs = Mat::Zero(tree[j][k].NumLocals, 1);
    }
}

void Tree::initialise_P2P_Leaf_Level() {  // T:3372-3386
  const int j = nLevels;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    for (int nn : tree[j][k].neighborList) tree[j][k].P2P[nn];
    tree[j][k].P2P[k];
  }
#pragma omp parallel for schedule(dynamic)
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    for (int nn : tree[j][k].neighborList)
      if (nn != k) tree[j][k].P2P[nn] = K->getMatrix(tree[j][k].chargeLocations, tree[j][nn].chargeLocations);
    tree[j][k].P2P[k] = K->getMatrix(tree[j][k].chargeLocations, tree[j][k].chargeLocations);
  }
}

void Tree::build() {  // AIFMM.cpp:7-93
  double t0 = now();
  createTree();
  assign_Center_Location();
  assign_Tree_Interactions();
  assignChargeLocations();
  assignNonLeafChargeLocations();
  getNodes();
  assemble_M2L();
  free_charge_and_checkPoints();
  initialise_phase();
  initialise_P2P_Leaf_Level();
  stats.tAssemble = now() - t0;
}

// ------------------------------------------------------------ non-leaf P2P
void Tree::initialise_P2P_NonLeafLevel(int j) {  // T:3413-3476
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    Box& B = tree[j][k];
    for (size_t n = 0; n < B.neighborList.size(); ++n) {
      int nn = B.neighborList[n];
      if (nn == k) continue;
      int n_rows = 0, n_cols = 0;
      for (int a = 0; a < nChild; ++a) {
        int t = 0;
        for (int b = 0; b < nChild; ++b) t += tree[j + 1][nChild * k + a].M2L[nChild * nn + b].c;
        n_cols = std::max(n_cols, t);
      }
      for (int b = 0; b < nChild; ++b) {
        int t = 0;
        for (int a = 0; a < nChild; ++a) t += tree[j + 1][nChild * k + a].M2L[nChild * nn + b].r;
        n_rows = std::max(n_rows, t);
      }
      B.P2P[nn] = Mat::Zero(n_rows, n_cols);
      int ri = 0, ci = 0;
      for (int a = 0; a < nChild; ++a) {
        for (int b = 0; b < nChild; ++b) {
          const Mat& m = tree[j + 1][nChild * k + a].M2L[nChild * nn + b];
          if (m.size() > 0) {
            B.P2P[nn].setBlock(ri, ci, m);
            ci += m.c;
          }
        }
        ri += tree[j + 1][nChild * k + a].M2L[nChild * nn + 0].r;
        ci = 0;
      }
    }
    {  // self
      int n_rows = 0, n_cols = 0;
      for (int a = 0; a < nChild; ++a) n_rows += tree[j + 1][nChild * k + a].NumLocals;
      for (int b = 0; b < nChild; ++b) n_cols += tree[j + 1][nChild * k + b].NumMultipoles;
      B.P2P[k] = Mat::Zero(n_rows, n_cols);
      int ri = 0, ci = 0;
      for (int a = 0; a < nChild; ++a) {
        for (int b = 0; b < nChild; ++b) {
          const Box& ca = tree[j + 1][nChild * k + a];
          const Box& cb = tree[j + 1][nChild * k + b];
          const Mat& m = tree[j + 1][nChild * k + a].M2L[nChild * k + b];
          if (m.r != ca.NumLocals || m.c != cb.NumMultipoles) fail("non-leaf self P2P block shape");
          B.P2P[k].setBlock(ri, ci, m);
          ci += cb.NumMultipoles;
        }
        ri += tree[j + 1][nChild * k + a].NumLocals;
        ci = 0;
      }
    }
  }
}

void Tree::deleteM2L(int j) {  // T:3478-3504
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    for (int nn : tree[j][k].neighborList) {
      if (nn == k) continue;
      for (int a = 0; a < nChild; ++a)
        for (int b = 0; b < nChild; ++b)
          if (tree[j + 1][nChild * k + a].M2L[nChild * nn + b].size() > 0)
            tree[j + 1][nChild * k + a].M2L[nChild * nn + b] = Mat(0, 0);
    }
    for (int a = 0; a < nChild; ++a)
      for (int b = 0; b < nChild; ++b) tree[j + 1][nChild * k + a].M2L[nChild * k + b] = Mat(0, 0);
  }
}

// ------------------------------------------------------------ recompression
bool Tree::is_well_separated(int j, int k, int l) {  // T:4044-4055
  if (k == l) return false;
  for (int nn : tree[j][k].neighborList)
    if (l == nn) return false;
  return true;
}

void Tree::update_other_M2Ls_at_k_old(int j, int k, int b, const Mat& nL2P) {  // T:3159-3188
  Box& B = tree[j][k];
  for (auto& kv : B.P2L) B.P2L[kv.first] = nL2P.adjoint() * B.L2P * B.P2L[kv.first];
  for (int kIL : B.interactionList) {
    if (kIL == b) continue;
    B.M2L[kIL] = nL2P.adjoint() * B.L2P * B.M2L[kIL];
  }
  for (int kN : B.neighborList)
    if ((kN != k) && tree[j][kN].Eliminated && B.Eliminated) B.M2L[kN] = nL2P.adjoint() * B.L2P * B.M2L[kN];
  if (B.Eliminated) B.M2L[k] = nL2P.adjoint() * B.L2P * B.M2L[k];
}

void Tree::update_other_M2Ls_at_b_old(int j, int k, int b, const Mat& nP2Mt) {  // T:3252-3288
  Box& Bb = tree[j][b];
  for (auto& kv : Bb.P2L) {
    int key = kv.first;
    tree[j][key].M2P[b] = tree[j][key].M2P[b] * Bb.P2M * nP2Mt;
  }
  for (int kIL : Bb.interactionList) {
    if (kIL == k) continue;
    tree[j][kIL].M2L[b] = tree[j][kIL].M2L[b] * Bb.P2M * nP2Mt;
  }
  for (int kN : Bb.neighborList)
    if (kN != b && tree[j][kN].Eliminated && Bb.Eliminated) tree[j][kN].M2L[b] = tree[j][kN].M2L[b] * Bb.P2M * nP2Mt;
  if (Bb.Eliminated) Bb.M2L[b] = Bb.M2L[b] * Bb.P2M * nP2Mt;
}

void Tree::update_parent_L2P_old(int j, int k, const Mat& nL2P) {  // T:3290-3314
  int kP = k / nChild, c_k = k % nChild;
  std::vector<Mat> U(nChild);
  int ri = 0;
  Mat& PL = tree[j - 1][kP].L2P;
  for (int c = 0; c < nChild; ++c) {
    U[c] = PL.block(ri, 0, tree[j][kP * nChild + c].NumLocals, PL.c);
    ri += tree[j][kP * nChild + c].NumLocals;
  }
  U[c_k] = nL2P.adjoint() * tree[j][k].L2P * U[c_k];
  int nr = 0;
  for (int c = 0; c < nChild; ++c) nr += U[c].r;
  Mat M(nr, U[0].c);
  ri = 0;
  for (int c = 0; c < nChild; ++c) {
    M.setBlock(ri, 0, U[c]);
    ri += U[c].r;
  }
  PL = M;
}

void Tree::update_parent_P2M_old(int j, int b, const Mat& nP2Mt) {  // T:3316-3340
  int bP = b / nChild, c_b = b % nChild;
  std::vector<Mat> V(nChild);
  int ci = 0;
  Mat& PM = tree[j - 1][bP].P2M;
  for (int c = 0; c < nChild; ++c) {
    V[c] = PM.block(0, ci, PM.r, tree[j][bP * nChild + c].NumMultipoles);
    ci += tree[j][bP * nChild + c].NumMultipoles;
  }
  V[c_b] = V[c_b] * tree[j][b].P2M * nP2Mt;
  int nc = 0;
  for (int c = 0; c < nChild; ++c) nc += V[c].c;
  Mat M(V[0].r, nc);
  ci = 0;
  for (int c = 0; c < nChild; ++c) {
    M.setBlock(0, ci, V[c]);
    ci += V[c].c;
  }
  PM = M;
}

void Tree::compress_P2P_myRRQR(int j, int k, int b, const Mat& old_L2P, const Mat& old_P2M, const Mat& P2Pt,
                               Mat& new_L2P, Mat& new_P2Mt, Mat& Rk, Mat& Rn, Mat& Rn_prime, Mat& newM2L) {
  // T:1573-1656
  Mat A_col = hcat(old_L2P, P2Pt);
  RRQRResult r1;
  rrqrPartition(A_col, TOL_POW, fill_in_TOL_POW, old_L2P.c, tree[j][k].maxPivot_L2P, fillin_rankVec[j], realMode, r1);
  stats.nRRQR++;
  tree[j][k].maxPivot_L2P = std::max(tree[j][k].maxPivot_L2P, r1.maxPivot);
  new_L2P = r1.Q;
  Rk = new_L2P.adjoint() * old_L2P;
  Mat Rk_prime = new_L2P.adjoint() * P2Pt;
  Mat A_row = hcat(old_P2M.adjoint(), Rk_prime.adjoint());
  RRQRResult r2;
  rrqrPartition(A_row, TOL_POW, fill_in_TOL_POW, old_P2M.r, tree[j][b].maxPivot_P2M, fillin_rankVec[j], realMode, r2);
  stats.nRRQR++;
  tree[j][b].maxPivot_P2M = std::max(tree[j][b].maxPivot_P2M, r2.maxPivot);
  new_P2Mt = r2.Q;
  Rn = new_P2Mt.adjoint() * old_P2M.adjoint();
  Rn_prime = new_P2Mt.adjoint() * Rk_prime.adjoint();
  if (tree[j][k].M2L[b].size() > 0) newM2L = (Rk * tree[j][k].M2L[b]) * Rn.adjoint() + Rn_prime.adjoint();
  else newM2L = Rn_prime.adjoint();
}

static void equalise(const Mat& L2P, const Mat& P2Mt, Mat& L2Pm, Mat& P2Mtm) {
  if (L2P.c < P2Mt.c) {
    P2Mtm = P2Mt.block(0, 0, P2Mt.r, L2P.c);
    L2Pm = L2P;
  } else {
    L2Pm = L2P.block(0, 0, L2P.r, P2Mt.c);
    P2Mtm = P2Mt;
  }
}

void Tree::compress_P2P_Two_Ways_myRRQR(int j, int k, int b) {  // T:2116-2306
  if (tree[j][b].M2L[k].size() == 0 || tree[j][k].M2L[b].size() == 0) return;
  stats.nCompressP2P++;
  Mat nL2P_k, nP2Mt_b, M2L_k_b, Rk, Rn, Rnp;
  {
    Mat a = tree[j][k].L2P, bb = tree[j][b].P2M, c = tree[j][k].P2P[b];
    compress_P2P_myRRQR(j, k, b, a, bb, c, nL2P_k, nP2Mt_b, Rk, Rn, Rnp, M2L_k_b);
  }
  Mat nL2P_b, nP2Mt_k, M2L_b_k;
  {
    Mat a = tree[j][b].L2P, bb = tree[j][k].P2M, c = tree[j][b].P2P[k];
    compress_P2P_myRRQR(j, b, k, a, bb, c, nL2P_b, nP2Mt_k, Rk, Rn, Rnp, M2L_b_k);
  }
  Mat nL2P_k_m, nP2Mt_k_m, nL2P_b_m, nP2Mt_b_m;
  equalise(nL2P_k, nP2Mt_k, nL2P_k_m, nP2Mt_k_m);
  equalise(nL2P_b, nP2Mt_b, nL2P_b_m, nP2Mt_b_m);
  tree[j][k].M2L[b] = M2L_k_b.block(0, 0, nL2P_k_m.c, nP2Mt_b_m.c);
  update_other_M2Ls_at_k_old(j, k, b, nL2P_k_m);
  update_other_M2Ls_at_b_old(j, k, b, nP2Mt_b_m);
  if (j > startLevel) {
    update_parent_L2P_old(j, k, nL2P_k_m);
    update_parent_P2M_old(j, b, nP2Mt_b_m);
  }
  tree[j][k].L2P = nL2P_k_m;
  tree[j][b].P2M = nP2Mt_b_m.adjoint();
  tree[j][k].NumLocals = tree[j][k].L2P.c;
  tree[j][b].NumMultipoles = tree[j][b].P2M.r;
  tree[j][b].M2L[k] = M2L_b_k.block(0, 0, nL2P_b_m.c, nP2Mt_k_m.c);
  update_other_M2Ls_at_k_old(j, b, k, nL2P_b_m);
  update_other_M2Ls_at_b_old(j, b, k, nP2Mt_k_m);
  if (j > startLevel) {
    update_parent_L2P_old(j, b, nL2P_b_m);
    update_parent_P2M_old(j, k, nP2Mt_k_m);
  }
  tree[j][b].L2P = nL2P_b_m;
  tree[j][k].P2M = nP2Mt_k_m.adjoint();
  tree[j][b].NumLocals = tree[j][b].L2P.c;
  tree[j][k].NumMultipoles = tree[j][k].P2M.r;
}

void Tree::compress_M2P_myRRQR(int j, int k, int b, Mat& nL2P, Mat& M2L) {  // T:2878-2902
  Box& B = tree[j][k];
  Mat A_col = hcat(B.L2P, B.M2P[b]);
  RRQRResult r;
  rrqrPartition(A_col, TOL_POW, fill_in_TOL_POW, B.L2P.c, B.maxPivot_L2P, fillin_rankVec[j], realMode, r);
  stats.nRRQR++;
  nL2P = r.Q;
  B.maxPivot_L2P = std::max(B.maxPivot_L2P, r.maxPivot);
  Mat Rk = nL2P.adjoint() * B.L2P;
  Mat Rkp = nL2P.adjoint() * B.M2P[b];
  M2L = Rk * B.M2L[b] + Rkp;
}

void Tree::compress_P2L_myRRQR(int j, int k, int b, Mat& nP2Mt, Mat& M2L) {  // T:2905-2959
  Box& Bb = tree[j][b];
  Mat A_row = hcat(Bb.P2M.adjoint(), tree[j][k].P2L[b].adjoint());
  RRQRResult r;
  rrqrPartition(A_row, TOL_POW, fill_in_TOL_POW, Bb.P2M.r, Bb.maxPivot_P2M, fillin_rankVec[j], realMode, r);
  stats.nRRQR++;
  nP2Mt = r.Q;
  Bb.maxPivot_P2M = std::max(Bb.maxPivot_P2M, r.maxPivot);
  Mat Rn = nP2Mt.adjoint() * Bb.P2M.adjoint();
  Mat Rnp = nP2Mt.adjoint() * tree[j][k].P2L[b].adjoint();
  M2L = tree[j][k].M2L[b] * Rn.adjoint() + Rnp.adjoint();
}

void Tree::compress_M2P_P2L_myRRQR(int j, int k, int b) {  // T:2454-2596
  if (tree[j][b].M2L[k].size() == 0 || tree[j][k].M2L[b].size() == 0) return;
  stats.nCompressP2L++;
  Mat nL2P_k, M2L_k_b;
  compress_M2P_myRRQR(j, k, b, nL2P_k, M2L_k_b);
  Mat nP2Mt_k, M2L_b_k;
  compress_P2L_myRRQR(j, b, k, nP2Mt_k, M2L_b_k);
  Mat nL2P_k_m, nP2Mt_k_m;
  equalise(nL2P_k, nP2Mt_k, nL2P_k_m, nP2Mt_k_m);
  tree[j][k].M2L[b] = M2L_k_b.block(0, 0, nL2P_k_m.c, M2L_k_b.c);
  update_other_M2Ls_at_k_old(j, k, b, nL2P_k_m);
  if (j > startLevel) update_parent_L2P_old(j, k, nL2P_k_m);
  tree[j][k].L2P = nL2P_k_m;
  tree[j][k].NumLocals = tree[j][k].L2P.c;
  tree[j][b].M2L[k] = M2L_b_k.block(0, 0, M2L_b_k.r, nP2Mt_k_m.c);
  update_other_M2Ls_at_b_old(j, b, k, nP2Mt_k_m);
  if (j > startLevel) update_parent_P2M_old(j, k, nP2Mt_k_m);
  tree[j][k].P2M = nP2Mt_k_m.adjoint();
  tree[j][k].NumMultipoles = tree[j][k].P2M.r;
}

// ------------------------------------------------------------ elimination
void Tree::eliminate_x(int j, int k) {  // T:3561-3611 with :3656-3791 and :3800-4042
  Box& B = tree[j][k];
  auto E = [&](int x) { return tree[j][x].Eliminated; };
  if (B.P2P[k].size() != 0) {
    LU lu(B.P2P[k]);
    B.L2M_f = -B.P2M * lu.solve(B.L2P);
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      if (!E(nn)) B.P2M_f[nn] = -B.P2M * lu.solve(B.P2P[nn]);
      else B.M2M_f[nn] = -B.P2M * lu.solve(B.M2P[nn]);
    }
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      Box& Bn = tree[j][nn];
      if (!E(nn)) Bn.L2P_f[k] = -Bn.P2P[k] * lu.solve(B.L2P);
      else Bn.L2P_f[k] = -Bn.P2L[k] * lu.solve(B.L2P);
      for (int pp : B.neighborList) {
        if (pp == k) continue;
        if (!E(nn)) {
          if (!E(pp)) {
            if (Bn.P2P[pp].size() == 0) Bn.P2P[pp] = -Bn.P2P[k] * lu.solve(B.P2P[pp]);
            else Bn.P2P[pp] = Bn.P2P[pp] - Bn.P2P[k] * lu.solve(B.P2P[pp]);
          } else {
            if (Bn.M2P[pp].size() == 0) Bn.M2P[pp] = -Bn.P2P[k] * lu.solve(B.M2P[pp]);
            else Bn.M2P[pp] = Bn.M2P[pp] - Bn.P2P[k] * lu.solve(B.M2P[pp]);
          }
        } else {
          if (!E(pp)) {
            if (Bn.P2L[pp].size() == 0) Bn.P2L[pp] = -Bn.P2L[k] * lu.solve(B.P2P[pp]);
            else Bn.P2L[pp] = Bn.P2L[pp] - Bn.P2L[k] * lu.solve(B.P2P[pp]);
          } else {
            if (Bn.M2L[pp].size() > 0) Bn.M2L[pp] = Bn.M2L[pp] - Bn.P2L[k] * lu.solve(B.M2P[pp]);
            else Bn.M2L[pp] = -Bn.P2L[k] * lu.solve(B.M2P[pp]);
          }
        }
      }
    }
  } else {
    B.L2M_f = Mat::Zero(B.P2M.r, B.L2P.c);
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      if (!E(nn)) B.P2M_f[nn] = Mat::Zero(B.P2M.r, B.P2P[nn].c);
      else B.M2M_f[nn] = Mat::Zero(B.P2M.r, B.M2P[nn].c);
    }
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      Box& Bn = tree[j][nn];
      if (!E(nn)) Bn.L2P_f[k] = Mat::Zero(Bn.P2P[k].r, B.L2P.c);
      else Bn.L2P_f[k] = Mat::Zero(Bn.P2L[k].r, B.L2P.c);
      for (int pp : B.neighborList) {
        if (pp == k) continue;
        if (!E(nn)) {
          if (!E(pp)) {
            if (Bn.P2P[pp].size() == 0) Bn.P2P[pp] = Mat::Zero(Bn.P2P[k].r, B.P2P[pp].c);
          } else {
            if (Bn.M2P[pp].size() == 0) Bn.M2P[pp] = Mat::Zero(Bn.P2P[k].r, B.M2P[pp].c);
          }
        } else {
          if (!E(pp)) {
            if (Bn.P2L[pp].size() == 0) Bn.P2L[pp] = Mat::Zero(Bn.P2L[k].r, B.P2P[pp].c);
          } else {
            Bn.M2L[pp];
          }
        }
      }
    }
  }
}

void Tree::eliminate_z(int j, int k) {  // T:4081-4113 with :4151-4296 and :4304-4509
  Box& B = tree[j][k];
  auto E = [&](int x) { return tree[j][x].Eliminated; };
  if (B.L2M_f.size() > 0) {
    LU lu(B.L2M_f);
    const Mat negI = -Mat::Identity(B.NumMultipoles, B.NumMultipoles);
    const Mat Xy = lu.solve(negI);
    B.M2L[k] = Xy;
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      if (!E(nn)) {
        B.P2L[nn] = lu.solve(B.P2M_f[nn]);
        if (is_well_separated(j, k, nn)) {
          if (B.M2L[nn].norm() > 0 && B.P2L[nn].norm() / B.M2L[nn].norm() != 0.0) P2L_M2P.push_back({k, nn});
        }
      } else {
        B.M2L[nn] = lu.solve(B.M2M_f[nn]);
      }
    }
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      Box& Bn = tree[j][nn];
      // filings_in_equation_P2P_due_to_y, T:4471-4509
      if (!E(nn)) {
        if (Bn.M2P[k].size() == 0) Bn.M2P[k] = -Bn.L2P_f[k] * lu.solve(negI);
        else Bn.M2P[k] = Bn.M2P[k] - Bn.L2P_f[k] * lu.solve(negI);
      } else {
        if (Bn.M2L[k].size() == 0) Bn.M2L[k] = -Bn.L2P_f[k] * lu.solve(negI);
        else Bn.M2L[k] = Bn.M2L[k] - Bn.L2P_f[k] * lu.solve(negI);
      }
      // filings_in_equation_P2P_due_to_neighbors, T:4399-4469
      for (int pp : B.neighborList) {
        if (pp == k) continue;
        if (!E(nn)) {
          if (!E(pp)) {
            Bn.P2P[pp] = Bn.P2P[pp] - Bn.L2P_f[k] * lu.solve(B.P2M_f[pp]);
            if (is_well_separated(j, nn, pp)) {
              if (nn < pp) {
                if (Bn.M2L[pp].norm() > 0 && Bn.P2P[pp].norm() / Bn.M2L[pp].norm() > fillInTolerance)
                  P2Pq.push_back({nn, pp});
              }
            }
          } else {
            Bn.M2P[pp] = Bn.M2P[pp] - Bn.L2P_f[k] * lu.solve(B.M2M_f[pp]);
          }
        } else {
          if (!E(pp)) {
            Bn.P2L[pp] = Bn.P2L[pp] - Bn.L2P_f[k] * lu.solve(B.P2M_f[pp]);
            if (is_well_separated(j, nn, pp)) {
              if (Bn.M2L[pp].norm() > 0 && Bn.P2L[pp].norm() / Bn.M2L[pp].norm() > fillInTolerance)
                P2L_M2P.push_back({nn, pp});
            }
          } else {
            Bn.M2L[pp] = Bn.M2L[pp] - Bn.L2P_f[k] * lu.solve(B.M2M_f[pp]);
          }
        }
      }
    }
  } else {
    B.M2L[k] = Mat::Zero(0, B.NumMultipoles);
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      if (!E(nn)) B.P2L[nn] = Mat::Zero(0, B.P2M_f[nn].c);
      else B.M2L[nn] = Mat::Zero(0, B.M2M_f[nn].c);
    }
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      Box& Bn = tree[j][nn];
      if (!E(nn)) {
        if (Bn.M2P[k].size() == 0) Bn.M2P[k] = Mat::Zero(Bn.L2P_f[k].r, B.NumMultipoles);
      } else {
        if (Bn.M2L[k].size() == 0) Bn.M2L[k] = Mat::Zero(Bn.L2P_f[k].r, B.NumMultipoles);
      }
      for (int pp : B.neighborList) {
        if (pp == k) continue;
        if (!E(nn)) {
          if (!E(pp)) Bn.P2P[pp];
          else Bn.M2P[pp];
        } else {
          if (!E(pp)) Bn.P2L[pp];
          else Bn.M2L[pp];
        }
      }
    }
  }
}

void Tree::factorize() {  // eliminate_phase_efficient, T:4599-4747
  double t0 = now();
  for (int j = nLevels; j >= startLevel; --j) {
    if (j != nLevels) {
      initialise_P2P_NonLeafLevel(j);
      deleteM2L(j);
    }
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      for (int i = 0; i < (int)P2Pq.size(); i++) {
        int nn = P2Pq[i].first, pp = P2Pq[i].second;
        if (k == nn || k == pp) {
          P2Pq.erase(P2Pq.begin() + i);
          i--;
          if (tree[j][nn].P2P[pp].size() != 0) {
            compress_P2P_Two_Ways_myRRQR(j, nn, pp);
            tree[j][nn].P2P[pp] = Mat(0, 0);
            tree[j][pp].P2P[nn] = Mat(0, 0);
          }
        }
      }
      for (int i = 0; i < (int)P2L_M2P.size(); i++) {
        int nn = P2L_M2P[i].first, pp = P2L_M2P[i].second;
        if (k == nn || k == pp) {
          P2L_M2P.erase(P2L_M2P.begin() + i);
          i--;
          if (tree[j][nn].P2L[pp].size() != 0) {
            compress_M2P_P2L_myRRQR(j, pp, nn);
            tree[j][nn].P2L[pp] = Mat(0, 0);
            tree[j][pp].M2P[nn] = Mat(0, 0);
          }
        }
      }
      tree[j][k].Eliminated = true;
      eliminate_x(j, k);
      eliminate_z(j, k);
    }
  }
  stats.tFactor = now() - t0;
}

// ------------------------------------------------------------ solve
void Tree::assign_Leaf_rhs(const Mat& charges) {  // T:670-678
  const int j = nLevels;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    Box& B = tree[j][k];
    B.particle_rhs = Mat::Zero((int)B.chargeLocations.size(), 1);
    for (size_t i = 0; i < B.chargeLocations.size(); ++i) B.particle_rhs(i) = charges(B.chargeLocations[i]);
  }
}

void Tree::assign_particle_rhs_NonLeafLevel(int j) {  // T:3506-3523
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    int len = 0;
    for (int c = 0; c < nChild; ++c) len += tree[j + 1][nChild * k + c].multipole_rhs.r;
    Mat v(len, 1);
    int o = 0;
    for (int c = 0; c < nChild; ++c) {
      const Mat& m = tree[j + 1][nChild * k + c].multipole_rhs;
      for (int i = 0; i < m.r; ++i) v(o + i) = m(i);
      o += m.r;
    }
    tree[j][k].particle_rhs = v;
  }
}

void Tree::rhs_eliminate_x(int j, int k) {  // T:3613-3653, :3795-3886
  Box& B = tree[j][k];
  if (B.P2P[k].size() != 0) {
    LU lu(B.P2P[k]);
    B.local_rhs = -B.P2M * lu.solve(B.particle_rhs);
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      Box& Bn = tree[j][nn];
      if (!Bn.Eliminated) Bn.particle_rhs = Bn.particle_rhs - Bn.P2P[k] * lu.solve(B.particle_rhs);
      else Bn.multipole_rhs = Bn.multipole_rhs - Bn.P2L[k] * lu.solve(B.particle_rhs);
    }
  } else {
    B.local_rhs = Mat::Zero(B.P2M.r, 1);
  }
}

void Tree::rhs_eliminate_z(int j, int k) {  // T:4115-4148, :4313-4397
  Box& B = tree[j][k];
  if (B.L2M_f.size() > 0) {
    LU lu(B.L2M_f);
    B.multipole_rhs = lu.solve(B.local_rhs);
    for (int nn : B.neighborList) {
      if (nn == k) continue;
      Box& Bn = tree[j][nn];
      if (!Bn.Eliminated) Bn.particle_rhs = Bn.particle_rhs - Bn.L2P_f[k] * lu.solve(B.local_rhs);
      else Bn.multipole_rhs = Bn.multipole_rhs - Bn.L2P_f[k] * lu.solve(B.local_rhs);
    }
  } else {
    B.multipole_rhs = Mat(0, 1);
  }
}

void Tree::rhs_eliminate_phase_efficient() {  // T:4749-4770
  for (int j = nLevels; j >= startLevel; --j)
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) tree[j][k].Eliminated = false;
  for (int j = nLevels; j >= startLevel; --j) {
    if (j != nLevels) assign_particle_rhs_NonLeafLevel(j);
    for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
      tree[j][k].Eliminated = true;
      rhs_eliminate_x(j, k);
      rhs_eliminate_z(j, k);
    }
  }
}

void Tree::solve_particles_at_base_level(int j) {  // T:4772-4810
  int NM = 0, NL = 0;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    NM += tree[j][k].NumMultipoles;
    NL += tree[j][k].NumLocals;
  }
  if (NL == 0 || NM == 0) return;
  Mat A = Mat::Zero(NL, NM);
  Mat b = Mat::Zero(NL, 1);
  int ri = 0;
  for (int r = 0; r < nBoxesPerLevel[j]; ++r) {
    int si = 0;
    for (int s = 0; s < nBoxesPerLevel[j]; ++s) {
      const Mat& m = tree[j][r].M2L[s];
      // Eigen's block assignment asserts on a shape mismatch; so does this.
      if (m.r != tree[j][r].NumLocals || m.c != tree[j][s].NumMultipoles) fail("base-level M2L block shape");
      A.setBlock(ri, si, m);
      si += tree[j][s].NumMultipoles;
    }
    const Mat& mr = tree[j][r].multipole_rhs;
    for (int i = 0; i < tree[j][r].NumLocals; ++i) b(ri + i) = mr(i);
    ri += tree[j][r].NumLocals;
  }
  if (NL != NM) fail("base-level system is not square");
  LU lu(A);
  Mat mp = lu.solve(b);
  int idx = 0;
  for (int k = 0; k < nBoxesPerLevel[j]; ++k) {
    tree[j][k].multipoles = mp.block(idx, 0, tree[j][k].NumMultipoles, 1);
    idx += tree[j][k].NumMultipoles;
  }
}

void Tree::back_substitution_phase() {  // T:4812-4865
  solve_particles_at_base_level(startLevel);
  for (int j = startLevel; j <= nLevels; j++) {
    for (int k = nBoxesPerLevel[j] - 1; k >= 0; k--) {
      Box& B = tree[j][k];
      if (B.P2P[k].size() != 0) {
        LU lu(B.P2P[k]);
        Mat rhs1 = B.particle_rhs;
        for (int nn : B.neighborList) {
          if (nn == k) continue;
          if (!tree[j][nn].Eliminated) rhs1 = rhs1 - B.P2P[nn] * tree[j][nn].particles;
          else rhs1 = rhs1 - B.M2P[nn] * tree[j][nn].multipoles;
        }
        Mat rhs2 = B.multipoles - B.P2M * lu.solve(rhs1);
        Mat Atemp = -B.P2M * lu.solve(B.L2P);
        if (Atemp.size() != 0) {
          LU la(Atemp);
          B.locals = la.solve(rhs2);
        } else {
          B.locals = Mat(0, 1);
        }
        B.particles = lu.solve(rhs1 - B.L2P * B.locals);
      } else {
        B.particles = Mat(0, 1);
      }
      B.Eliminated = false;
      if (nLevels != j) {
        int idx = 0;
        for (int c = 0; c < nChild; ++c) {
          Box& C = tree[j + 1][nChild * k + c];
          C.multipoles = B.particles.block(idx, 0, C.NumMultipoles, 1);
          idx += C.NumMultipoles;
        }
      }
    }
  }
}

void Tree::getx(Mat& x) {  // T:4874-4907
  x = Mat::Zero(N, 1);
  int idx = 0;
  for (int k = 0; k < nBoxesPerLevel[nLevels]; ++k) {
    const Box& B = tree[nLevels][k];
    for (int i = 0; i < B.particles.r; ++i) x(idx + i) = B.particles(i);
    idx += (int)B.chargeLocations.size();
  }
}

void Tree::reorder(Mat& x) {  // T:466-476
  Mat t = x;
  int start = 0;
  for (int k = 0; k < nBoxesPerLevel[nLevels]; ++k)
    for (int index : tree[nLevels][k].chargeLocations) x(index) = t(start++);
}

void Tree::solve(const Mat& rhs, Mat& x) {
  double t0 = now();
  assign_Leaf_rhs(rhs);
  rhs_eliminate_phase_efficient();
  back_substitution_phase();
  stats.tSolve = now() - t0;
  getx(x);
  reorder(x);
}

// ------------------------------------------------------------ diagnostics
int Tree::getAvgLeafSize() const {  // T:490-501
  int avg = 0, nBox = 0;
  for (const Box& B : tree[nLevels])
    if (B.chargeLocations.size() > 0) {
      nBox++;
      avg += (int)B.chargeLocations.size();
    }
  return nBox ? avg / nBox : 0;
}

int Tree::getAvgMultipoles() const {  // T:531-552 (prints dropped)
  int avg = 0, nBox = 0;
  for (int j = nLevels; j >= startLevel; j--)
    for (const Box& B : tree[j])
      if (B.P2M.r > 0 && B.interactionList.size() > 0) {
        nBox++;
        avg += B.P2M.r;
      }
  return nBox ? avg / nBox : 0;
}

int Tree::maxRank() const {
  int mx = 0;
  for (int j = nLevels; j >= startLevel; j--)
    for (const Box& B : tree[j]) mx = std::max(mx, B.P2M.r);
  return mx;
}

double Tree::findMemory() {  // T:4511-4539
  double sum = 0.0;
  for (int j = nLevels; j >= startLevel; --j)
    for (Box& B : tree[j]) sum += B.L2P.size() + B.P2M.size();
  for (int j = nLevels; j >= startLevel; --j)
    for (Box& B : tree[j])
      for (int n : B.interactionList) sum += B.M2L[n].size();
  for (Box& B : tree[nLevels])
    for (int n : B.neighborList) sum += B.P2P[n].size();
  return sum * 8 * 1e-9;
}

double Tree::findMemoryAfterFactorize() {  // T:4541-4571
  double sum = 0.0;
  for (int j = nLevels; j >= startLevel; --j)
    for (Box& B : tree[j]) sum += B.L2P.size() + B.P2M.size();
  for (int j = nLevels; j >= startLevel; --j)
    for (Box& B : tree[j])
      for (int n : B.neighborList) sum += B.P2P[n].size();
  return sum * 8 * 1e-9;
}

}  // namespace orc
