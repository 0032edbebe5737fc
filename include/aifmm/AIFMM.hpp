// Drop-in replacement for the reference's include/AIFMM.hpp: the solver
// facade AIFMM<kerneltype> (include/AIFMM.hpp:11-36, src/AIFMM.cpp:7-167),
// header-only over libaifmm_b200.  AIFMM<EFIEMatrix> and
// AIFMM<ElectrostaticsMatrix> work; any kerneltype derived from `kernel` whose
// `handle` is set by the library does.
//
// As in the reference, solve() returns the solution in TREE order (getx
// without reorder, src/AIFMM.cpp:102-110) and getPhi() in unknown order.
#ifndef AIFMM_DROPIN_AIFMM_HPP
#define AIFMM_DROPIN_AIFMM_HPP

#include "AIFMMTree.hpp"
#include "EFIEMatrix.hpp"
#include "ElectrostaticsMatrix.hpp"

template <typename kerneltype>
class AIFMM {
 public:
  FMM2DTree<kerneltype>* A;

  // tree, skeletons, M2L and leaf P2P blocks (AIFMM.cpp:7-93)
  AIFMM(inputsToSolverClass inputsToSolver, kerneltype* mykernel)
      : A(new FMM2DTree<kerneltype>(inputsToSolver, mykernel)) {}
  AIFMM(const AIFMM&) = delete;
  AIFMM& operator=(const AIFMM&) = delete;

  void factorize() { A->eliminate_phase_efficient(); }

  Vec solve(Vec& rhs) {
    A->assign_Leaf_rhs(rhs);
    A->rhs_eliminate_phase_efficient();
    A->back_substitution_phase();
    Vec phi;
    A->getx(phi);
    return phi;
  }
  void backSubstitute(Vec& rhs) {
    A->assign_Leaf_rhs(rhs);
    A->rhs_eliminate_phase_efficient();
    A->back_substitution_phase();
  }
  void backSubstitute1(Vec& rhs) { A->assign_Leaf_rhs(rhs); }
  void backSubstitute2() { A->rhs_eliminate_phase_efficient(); }
  void backSubstitute3() { A->back_substitution_phase(); }
  void getPhi(Vec& phi) {
    A->getx(phi);
    A->reorder(phi);
  }
  void viewRankStructure(std::string filename) { A->viewRankStructure(filename); }

  ~AIFMM() { delete A; }
};

#endif
