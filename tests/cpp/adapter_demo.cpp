// Drives libmpdg through the C++ adapter (include/mpdg_operator.hpp) the way a
// MeltPoolDG operation drives OperatorMatrixFree: vmult, inverse diagonal and a
// CG + Jacobi solve on a host vector type.  Reads vertices, mask and src from
// a binary file, writes dst, the inverse diagonal and the solution.
//   adapter_demo <in.bin> <out.bin>
// in.bin:  int32 nc[3], int32 degree, int64 n_dofs, double vertices[3*nv],
//          uint8 mask[n_dofs], double src[n_dofs]
// out.bin: double dst[n_dofs], double inv_diag[n_dofs], double x[n_dofs], int32 iterations
#include <cstdio>
#include <fstream>
#include <vector>

#include "mpdg_operator.hpp"

struct HostVector {
  std::vector<double> v;
  explicit HostVector(size_t n) : v(n, 0.0) {}
  double *begin() { return v.data(); }
  const double *begin() const { return v.data(); }
  size_t size() const { return v.size(); }
};

int main(int argc, char **argv)
{
  if (argc != 3) return 2;
  std::ifstream in(argv[1], std::ios::binary);
  int nc[3], degree;
  int64_t n;
  in.read(reinterpret_cast<char *>(nc), sizeof(nc));
  in.read(reinterpret_cast<char *>(&degree), sizeof(degree));
  in.read(reinterpret_cast<char *>(&n), sizeof(n));
  const size_t nv = (size_t)(nc[0] + 1) * (nc[1] + 1) * (nc[2] + 1);
  std::vector<double> vert(3 * nv);
  std::vector<uint8_t> mask(n);
  HostVector src(n), dst(n), diag(n), x(n);
  in.read(reinterpret_cast<char *>(vert.data()), sizeof(double) * vert.size());
  in.read(reinterpret_cast<char *>(mask.data()), n);
  in.read(reinterpret_cast<char *>(src.begin()), sizeof(double) * n);
  try {
    mpdg::Mesh mesh(degree, nc, vert, mask);
    mpdg_op_desc d{};
    d.kind = MPDG_OP_HEAT;
    d.dt = 1e-3;
    d.rho_cp = 1.0;
    d.k0 = 1.0;
    mpdg::MatrixFreeOperator<HostVector> op(mesh, d);
    op.vmult(dst, src);
    op.compute_inverse_diagonal_from_matrixfree(diag);
    mpdg_solver_desc sd;
    mpdg_solver_desc_default(&sd);
    sd.solver = MPDG_SOLVER_CG;
    sd.rel_tolerance = 1e-10;
    const int it = op.solve(x, dst, sd);  // A x = A src  ->  x = src on the free DoFs
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char *>(dst.begin()), sizeof(double) * n);
    out.write(reinterpret_cast<const char *>(diag.begin()), sizeof(double) * n);
    out.write(reinterpret_cast<const char *>(x.begin()), sizeof(double) * n);
    out.write(reinterpret_cast<const char *>(&it), sizeof(it));
  } catch (const mpdg::Exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
