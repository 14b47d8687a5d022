// ORACLE — test infrastructure only.  The CPU build of the reference checker
// links CUP2D's ExpAMRSolver.cpp and LocalSpMatDnVec.cpp unchanged; this file
// defines the BiCGSTABSolver members those two call (declared in the
// reference's source/Poisson/BiCGSTAB.cuh) so that no GPU is needed.  Instead
// of uploading and solving, they record P^-1 and the assembled system, which
// BiCGSTABSolver may read as LocalSpMatDnVec's friend.  The GPU build links
// the reference's own BiCGSTAB.cu in place of this file.
#include "BiCGSTAB.cuh"
#include "ref_capture.hpp"

BiCGSTABSolver::BiCGSTABSolver(MPI_Comm m_comm, LocalSpMatDnVec& LocalLS, const int BLEN,
                               const bool bMeanConstraint, const std::vector<double>& P_inv)
    : m_comm_(m_comm), BLEN_(BLEN), bMeanConstraint_(bMeanConstraint), LocalLS_(LocalLS), prof_(m_comm) {
  MPI_Comm_rank(m_comm_, &rank_);
  MPI_Comm_size(m_comm_, &comm_size_);
  ref_capture().pinv = P_inv;
}

BiCGSTABSolver::~BiCGSTABSolver() {}

void BiCGSTABSolver::solveWithUpdate(const double, const double, const int) {
  RefCapture& c = ref_capture();
  c.m = LocalLS_.m_;
  c.mean_row = LocalLS_.bMeanRow_;
  c.row = LocalLS_.loc_cooRowA_int_;
  c.col = LocalLS_.loc_cooColA_int_;
  c.val = LocalLS_.loc_cooValA_;
  c.b = LocalLS_.b_;
  c.x0 = LocalLS_.x_;
  c.h2 = LocalLS_.h2_;
  c.have_system = true;
}

void BiCGSTABSolver::solveNoUpdate(const double, const double, const int) {
  RefCapture& c = ref_capture();
  c.b = LocalLS_.b_;
  c.x0 = LocalLS_.x_;
}
