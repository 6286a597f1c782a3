// mpdg_operator.hpp -- header-only C++ adapter that gives libmpdg's C ABI the
// shape of MeltPoolDG's matrix-free operator interface
// (include/meltpooldg/core/operator_base.hpp:189-283, OperatorMatrixFree):
//
//   vmult(dst, src)                                   operator_base.hpp:239-243
//   create_rhs(dst, src)                              operator_base.hpp:208-212
//   compute_inverse_diagonal_from_matrixfree(diag)    operator_base.hpp:268-272
//   reset_time_increment(dt)                          operator_base.hpp:41-46
//   reset_dof_index(with_dirichlet)                   operator_base.hpp:31-35
//
// VectorType is any host vector with `double *begin()`, `const double *begin()
// const` and `size()` in the library's lexicographic DoF numbering (for
// dealii::LinearAlgebra::distributed::Vector<double> on one rank these exist).
// Host vectors are copied to the device inside each call (the *_host entry
// points), so the adapter needs no CUDA headers.  Code that keeps its vectors
// on the device calls the device entry points (mpdg_vmult, mpdg_solve) with
// device pointers instead.
//
// Errors become exceptions of type mpdg::Exception, the counterpart of the
// reference's AssertThrow/ExcMessage; a solver that hits its iteration limit
// throws mpdg::NoConvergence (dealii::SolverControl::NoConvergence).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "mpdg.h"

namespace mpdg {

class Exception : public std::runtime_error {
 public:
  Exception(int status, const std::string &where)
      : std::runtime_error(where + ": status " + std::to_string(status) + ": " + mpdg_last_error()),
        status(status)
  {
  }
  int status;
};

class NoConvergence : public Exception {
 public:
  using Exception::Exception;
};

inline void check(int status, const char *where)
{
  if (status == MPDG_ERR_NOT_CONVERGED) throw NoConvergence(status, where);
  if (status != MPDG_OK) throw Exception(status, where);
}

// Owns a device mesh (the ScratchData/MatrixFree set-up of the reference).
class Mesh {
 public:
  Mesh(int degree, const int nc[3], const std::vector<double> &vertices,
       const std::vector<uint8_t> &dirichlet_mask = {})
  {
    mpdg_mesh_desc d{};
    d.dim = 3;
    d.degree = degree;
    for (int i = 0; i < 3; ++i) d.nc[i] = nc[i];
    d.vertices = vertices.data();
    d.dirichlet_mask = dirichlet_mask.empty() ? nullptr : dirichlet_mask.data();
    d.geometry = MPDG_GEOM_AUTO;
    check(mpdg_mesh_create(&d, &h_), "mpdg_mesh_create");
    check(mpdg_mesh_n_dofs(h_, &n_dofs_), "mpdg_mesh_n_dofs");
  }
  ~Mesh() { mpdg_mesh_destroy(h_); }
  Mesh(const Mesh &) = delete;
  Mesh &operator=(const Mesh &) = delete;
  mpdg_mesh *handle() const { return h_; }
  int64_t n_dofs() const { return n_dofs_; }

 private:
  mpdg_mesh *h_ = nullptr;
  int64_t n_dofs_ = 0;
};

// The operator with OperatorMatrixFree's methods.
template <typename VectorType>
class MatrixFreeOperator {
 public:
  MatrixFreeOperator(Mesh &mesh, const mpdg_op_desc &desc) : mesh_(mesh)
  {
    check(mpdg_op_create(mesh.handle(), &desc, &h_), "mpdg_op_create");
  }
  ~MatrixFreeOperator() { mpdg_op_destroy(h_); }
  MatrixFreeOperator(const MatrixFreeOperator &) = delete;
  MatrixFreeOperator &operator=(const MatrixFreeOperator &) = delete;

  void reset_time_increment(double dt) { check(mpdg_op_reset_time_increment(h_, dt), "reset_time_increment"); }
  void reset_dof_index(bool with_dirichlet) { check(mpdg_op_use_dirichlet(h_, with_dirichlet ? 1 : 0), "reset_dof_index"); }

  // state the operator reads (temperature for k(T) and the Newton residual);
  // host values are copied into operator-owned device memory
  void set_temperature(const VectorType &T)
  {
    size_check(T);
    check(mpdg_op_set_field_host(h_, MPDG_FIELD_TEMPERATURE, T.begin()), "set_field");
  }

  void vmult(VectorType &dst, const VectorType &src) const
  {
    size_check(dst);
    size_check(src);
    check(mpdg_vmult_host(h_, dst.begin(), src.begin()), "vmult");
  }

  // the reference inverts the diagonal in place on a dof vector
  void compute_inverse_diagonal_from_matrixfree(VectorType &diag) const
  {
    size_check(diag);
    check(mpdg_compute_inverse_diagonal_host(h_, diag.begin()), "compute_inverse_diagonal");
  }

  // dst += rhs contribution; heat: src = T_old (heat_source may be null),
  // advection-diffusion: src = phi_old
  void create_rhs(VectorType &dst, const VectorType &src, const VectorType *heat_source = nullptr) const
  {
    size_check(dst);
    size_check(src);
    if (heat_source) size_check(*heat_source);
    check(mpdg_create_rhs_host(h_, dst.begin(), src.begin(), heat_source ? heat_source->begin() : nullptr),
          "create_rhs");
  }

  // LinearSolver::solve: returns the iteration count
  int solve(VectorType &x, const VectorType &b, const mpdg_solver_desc &data) const
  {
    size_check(x);
    size_check(b);
    mpdg_solve_report rep{};
    check(mpdg_solve_host(h_, &data, x.begin(), b.begin(), &rep), "LinearSolver::solve");
    return rep.iterations;
  }

  mpdg_op *handle() const { return h_; }

 private:
  void size_check(const VectorType &v) const
  {
    if ((int64_t)v.size() != mesh_.n_dofs()) throw Exception(MPDG_ERR_ARG, "vector size");
  }

  Mesh &mesh_;
  mpdg_op *h_ = nullptr;
};

}  // namespace mpdg
