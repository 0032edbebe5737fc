// Checks of the Eigen subset under include/aifmm/Eigen against values worked
// out by hand.  Prints one line per failed check and exits 1 if any failed.
#include <Eigen/Dense>
#include <complex>
#include <iostream>
#include <sstream>

using namespace Eigen;
static int fails = 0;
#define CHECK(c)                                                       \
  do {                                                                 \
    if (!(c)) {                                                        \
      std::cout << "FAILED line " << __LINE__ << ": " #c << std::endl; \
      ++fails;                                                         \
    }                                                                  \
  } while (0)

int main() {
  typedef std::complex<double> cd;
  // shapes and element access, column-major storage
  MatrixXd M(3, 2);
  M(0, 0) = 1; M(1, 0) = 2; M(2, 0) = 3; M(0, 1) = -4; M(1, 1) = 5; M(2, 1) = 0.5;
  CHECK(M.rows() == 3 && M.cols() == 2 && M.size() == 6);
  CHECK(M.data()[1] == 2 && M.data()[3] == -4);
  // colwise reductions assigned to a column vector (transposed, as Eigen does)
  VectorXd mx = M.colwise().maxCoeff(), mn = M.colwise().minCoeff();
  CHECK(mx.rows() == 2 && mx.cols() == 1 && mx(0) == 3 && mx(1) == 5);
  CHECK(mn(0) == 1 && mn(1) == -4);
  // row assignment from a 3-vector expression
  Vector3d a(1, 2, 3), b(3, 2, 1);
  MatrixXd P(2, 3);
  P.row(0) = (a + b) / 2.0;
  P.row(1) = a.cross(b);
  CHECK(P(0, 0) == 2 && P(0, 1) == 2 && P(0, 2) == 2);
  CHECK(P(1, 0) == -4 && P(1, 1) == 8 && P(1, 2) == -4);
  // column assignment, vector arithmetic, norm
  VectorXd v(3);
  v(0) = 3; v(1) = 0; v(2) = 4;
  CHECK(v.norm() == 5.0 && v.squaredNorm() == 25.0);
  MatrixXd S(3, 2);
  S.col(0) = v;
  S.col(1) = 2.0 * v - v;
  CHECK(S(2, 0) == 4 && S(2, 1) == 4);
  // complex: dot is conjugate-linear in the first argument
  VectorXcd x(2), y(2);
  x(0) = cd(0, 1); x(1) = cd(1, 0);
  y(0) = cd(0, 1); y(1) = cd(2, 0);
  CHECK(x.dot(y) == cd(3, 0));
  VectorXcd z = VectorXcd::Zero(2);
  z = z + cd(0, 2) * x;
  CHECK(z(0) == cd(-2, 0) && z(1) == cd(0, 2));
  CHECK(std::abs(z.norm() - std::sqrt(8.0)) < 1e-15);
  // real vector times complex scalar gives a complex vector
  Vector3cd w = a * std::exp(cd(0, 0));
  CHECK(w(2) == cd(3, 0));
  // products and adjoint
  MatrixXcd A(2, 2);
  A(0, 0) = cd(1, 1); A(0, 1) = 2; A(1, 0) = 0; A(1, 1) = cd(0, -1);
  MatrixXcd AH = A.adjoint();
  CHECK(AH(0, 0) == cd(1, -1) && AH(1, 0) == cd(2, 0) && AH(1, 1) == cd(0, 1));
  MatrixXcd AA = A * AH;
  CHECK(AA(0, 0) == cd(6, 0) && AA(0, 1) == cd(0, 2) && AA(1, 1) == cd(1, 0));
  // blocks and segments
  MatrixXd B = MatrixXd::Zero(4, 4);
  B.block(1, 1, 2, 2) = MatrixXd::Identity(2, 2);
  CHECK(B(1, 1) == 1 && B(2, 2) == 1 && B(1, 2) == 0 && B(0, 0) == 0);
  VectorXd s = VectorXd::Zero(5);
  s.segment(1, 3) = v;
  CHECK(s(0) == 0 && s(1) == 3 && s(3) == 4 && s(4) == 0);
  // comma initializer fills row by row
  Matrix3d C;
  C << 1, 2, 3,
       4, 5, 6,
       7, 8, 9;
  CHECK(C(0, 1) == 2 && C(1, 0) == 4 && C(2, 2) == 9);
  // Eigen's default text layout: one row per line, columns right-aligned
  MatrixXd T(2, 2);
  T(0, 0) = 1; T(0, 1) = 10; T(1, 0) = 100; T(1, 1) = 2;
  std::ostringstream os;
  os << T;
  CHECK(os.str() == "  1  10\n100   2");
  // size errors throw instead of writing out of bounds
  bool threw = false;
  try {
    MatrixXd bad(2, 2);
    bad.row(0) = v;  // 3 entries into a row of 2
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  CHECK(threw);
  if (fails == 0) std::cout << "OK" << std::endl;
  return fails ? 1 : 0;
}
