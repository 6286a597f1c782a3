// Mapped meshes: the ingestion form of an unstructured hexahedral mesh.
// Included by operator_kernels.cu inside namespace mpdg, after the block
// kernels and their launchers.
//
// A host that owns its mesh (a deal.II DoFHandler / MatrixFree layout) hands
// over each cell's 8 corners and its cell->DoF map (n^3 global DoFs per cell,
// lexicographic within the cell), a Dirichlet mask and its homogeneous affine
// constraints (hanging nodes: x_c = sum_e w_e x_{m_e}, masters unconstrained).
//  * Cells are coloured greedily so that no two cells of a colour share a DoF;
//    the block cell kernel runs colour by colour and reads/writes through the
//    map, so the scatter needs no atomics and sums in a fixed order.
//  * The operator is sum_K C_K^T A_K C_K (read_dof_values /
//    distribute_local_to_global with constraints, heat_diffuse_operator.cpp:
//    199-241): the constrained entries of the operand are replaced by their
//    constraint (in a copy), the cells apply, and every master then adds its
//    constrained DoFs' rows in a fixed order (one thread per master: no
//    atomics) before those rows are zeroed.
//  * The diagonal of the cells that touch no constrained DoF comes from the
//    separable diag_kernel; the cells that do get their element matrices by
//    quadrature, and each DoF of such a cell adds w^T A_K w for its weight
//    vector w over the cell's local DoFs (the constraint weights through which
//    it enters), one warp per (cell, DoF) in a fixed order.

// ---------------------------------------------------------------- kernels

template <typename Real>
__global__ void cons_distribute_kernel(const Real *src, Real *tmp, long n_cons, const long *cdof, const long *ptr,
                                       const long *mast, const double *w, const uint8_t *dmask)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_cons) return;
  Real s = 0;
  for (long e = ptr[t]; e < ptr[t + 1]; ++e) {
    const long m = mast[e];
    if (!(dmask && dmask[m])) s += (Real)w[e] * src[m];
  }
  tmp[cdof[t]] = s;
}

template <typename Real>
__global__ void cons_condense_kernel(Real *dst, long n_masters, const long *mdof, const long *mptr,
                                     const long *mcons, const double *mw, const uint8_t *dmask)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_masters) return;
  const long m = mdof[t];
  if (dmask && dmask[m]) return;
  Real s = 0;
  for (long e = mptr[t]; e < mptr[t + 1]; ++e) s += (Real)mw[e] * dst[mcons[e]];
  dst[m] += s;
}

template <typename Real>
__global__ void cons_zero_kernel(Real *dst, long n_cons, const long *cdof)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n_cons) dst[cdof[t]] = Real(0);
}

// element matrices of the listed cells by quadrature:
// A(t,u) = sum_q c_mass JxW phi_t phi_u + phi_t c_vel b.grad phi_u + grad phi_t^T (c_diff G) grad phi_u
// (reference gradients; JxW and G = JxW J^-1 J^-T from the metric, b = JxW J^-1 u)
template <int P>
__global__ void elem_matrix_kernel(const KP<double> p, const long *ccells, double *A)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  const Tables<double> &T = tab<double>(P);
  const long cell = ccells[blockIdx.x];
  const double *m = p.metric + cell * metric_stride(n);
  const double *vb = p.velb ? p.velb + cell * velb_stride(n) : nullptr;
  double *Ac = A + (long)blockIdx.x * n3 * n3;
  for (int e = threadIdx.x; e < n3 * n3; e += blockDim.x) {
    const int t = e / n3, u = e % n3;
    const int tx = t % n, ty = (t / n) % n, tz = t / n2;
    const int ux = u % n, uy = (u / n) % n, uz = u / n2;
    double s = 0.0;
    for (int q = 0; q < n3; ++q) {
      const int qx = q % n, qy = (q / n) % n, qz = q / n2;
      const double st[3] = {T.S[qx * n + tx], T.S[qy * n + ty], T.S[qz * n + tz]};
      const double dt[3] = {T.D[qx * n + tx], T.D[qy * n + ty], T.D[qz * n + tz]};
      const double su[3] = {T.S[qx * n + ux], T.S[qy * n + uy], T.S[qz * n + uz]};
      const double du[3] = {T.D[qx * n + ux], T.D[qy * n + uy], T.D[qz * n + uz]};
      const double pt = st[0] * st[1] * st[2], pu = su[0] * su[1] * su[2];
      const double gt[3] = {dt[0] * st[1] * st[2], st[0] * dt[1] * st[2], st[0] * st[1] * dt[2]};
      const double gu[3] = {du[0] * su[1] * su[2], su[0] * du[1] * su[2], su[0] * su[1] * du[2]};
      const double JxW = m[q], G00 = m[n3 + q], G01 = m[2 * n3 + q], G02 = m[3 * n3 + q],
                   G11 = m[4 * n3 + q], G12 = m[5 * n3 + q], G22 = m[6 * n3 + q];
      double v = p.c_mass * JxW * pt * pu;
      if (vb) v += pt * p.c_vel * (vb[q] * gu[0] + vb[n3 + q] * gu[1] + vb[2 * n3 + q] * gu[2]);
      const double f0 = G00 * gu[0] + G01 * gu[1] + G02 * gu[2];
      const double f1 = G01 * gu[0] + G11 * gu[1] + G12 * gu[2];
      const double f2 = G02 * gu[0] + G12 * gu[1] + G22 * gu[2];
      v += p.c_diff * (gt[0] * f0 + gt[1] * f1 + gt[2] * f2);
      s += v;
    }
    Ac[e] = s;
  }
}

// element matrices of the listed cells of a heat operator whose coefficients
// follow the fields (k(T), the phase laws, the full Newton tangent;
// heat_diffuse_operator.cpp:1029-1078): the fields (read plain through the
// map, as read_dof_values_plain does) are interpolated to the Gauss points
// and the law evaluated there once per cell, then
// A(t,u) = sum_q phi_t [c_m JxW phi_u + c_v b.grad phi_u
//                       + (d c_m/dT (T - T_old) JxW + d c_v/dT b.grad T) phi_u]
//          + grad phi_t . [k G grad phi_u + dk/dT phi_u G grad T]
// (the bracketed Newton terms with the full tangent; reference gradients,
// G = JxW J^-1 J^-T, b = JxW J^-1 u)
template <int P>
__global__ void elem_matrix_field_kernel(const KP<double> p, const long *cells, double *A)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  const Tables<double> &T = tab<double>(P);
  __shared__ double sT[n3], sg[3][n3], sc[6][n3];  // T, reference grad T, (cm, cv, k, dcm, dcv, dk)
  const long cell = cells[blockIdx.x];
  const int *cmap = p.cmap + cell * n3;
  for (int q = threadIdx.x; q < n3; q += blockDim.x) {
    const int qc[3] = {q % n, (q / n) % n, q / n2};
    double tq = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, oq = 0.0, hq = 0.0;
    for (int t = 0; t < n3; ++t) {
      const int tc[3] = {t % n, (t / n) % n, t / n2};
      const double s0 = T.S[qc[0] * n + tc[0]], s1 = T.S[qc[1] * n + tc[1]], s2 = T.S[qc[2] * n + tc[2]];
      const double d0 = T.D[qc[0] * n + tc[0]], d1 = T.D[qc[1] * n + tc[1]], d2 = T.D[qc[2] * n + tc[2]];
      const long g = cmap[t];
      const double Tv = p.T[g];
      tq += s0 * s1 * s2 * Tv;
      g0 += d0 * s1 * s2 * Tv;
      g1 += s0 * d1 * s2 * Tv;
      g2 += s0 * s1 * d2 * Tv;
      if (p.Told) oq += s0 * s1 * s2 * p.Told[g];
      if (p.Hs) hq += s0 * s1 * s2 * p.Hs[g];
    }
    double cm, cv, kq, dcm, dcv, dk;
    law_eval<double>(p, tq, hq, cm, cv, kq, dcm, dcv, dk);
    sT[q] = tq - oq;  // T - T_old (the Newton term's increment)
    sg[0][q] = g0;
    sg[1][q] = g1;
    sg[2][q] = g2;
    sc[0][q] = cm;
    sc[1][q] = cv;
    sc[2][q] = kq;
    sc[3][q] = dcm;
    sc[4][q] = dcv;
    sc[5][q] = dk;
  }
  __syncthreads();
  const double *m = p.metric + cell * metric_stride(n);
  const double *vb = p.velb ? p.velb + cell * velb_stride(n) : nullptr;
  const bool newton = p.full_tangent != 0, incr = p.Told != nullptr;
  double *Ac = A + (long)blockIdx.x * n3 * n3;
  for (int e = threadIdx.x; e < n3 * n3; e += blockDim.x) {
    const int t = e / n3, u = e % n3;
    const int tc[3] = {t % n, (t / n) % n, t / n2}, uc[3] = {u % n, (u / n) % n, u / n2};
    double s = 0.0;
    for (int q = 0; q < n3; ++q) {
      const int qc[3] = {q % n, (q / n) % n, q / n2};
      double st[3], dt[3], su[3], du[3];
      for (int d = 0; d < 3; ++d) {
        st[d] = T.S[qc[d] * n + tc[d]];
        dt[d] = T.D[qc[d] * n + tc[d]];
        su[d] = T.S[qc[d] * n + uc[d]];
        du[d] = T.D[qc[d] * n + uc[d]];
      }
      const double pt = st[0] * st[1] * st[2], pu = su[0] * su[1] * su[2];
      const double gt[3] = {dt[0] * st[1] * st[2], st[0] * dt[1] * st[2], st[0] * st[1] * dt[2]};
      const double gu[3] = {du[0] * su[1] * su[2], su[0] * du[1] * su[2], su[0] * su[1] * du[2]};
      const double JxW = m[q], G00 = m[n3 + q], G01 = m[2 * n3 + q], G02 = m[3 * n3 + q],
                   G11 = m[4 * n3 + q], G12 = m[5 * n3 + q], G22 = m[6 * n3 + q];
      const double b0 = vb ? vb[q] : 0.0, b1 = vb ? vb[n3 + q] : 0.0, b2 = vb ? vb[2 * n3 + q] : 0.0;
      double fu0 = G00 * gu[0] + G01 * gu[1] + G02 * gu[2];
      double fu1 = G01 * gu[0] + G11 * gu[1] + G12 * gu[2];
      double fu2 = G02 * gu[0] + G12 * gu[1] + G22 * gu[2];
      double v = sc[0][q] * JxW * pu + sc[1][q] * (b0 * gu[0] + b1 * gu[1] + b2 * gu[2]);
      double f0 = sc[2][q] * fu0, f1 = sc[2][q] * fu1, f2 = sc[2][q] * fu2;
      if (newton) {
        const double du_ = sc[5][q] * pu;
        f0 += du_ * (G00 * sg[0][q] + G01 * sg[1][q] + G02 * sg[2][q]);
        f1 += du_ * (G01 * sg[0][q] + G11 * sg[1][q] + G12 * sg[2][q]);
        f2 += du_ * (G02 * sg[0][q] + G12 * sg[1][q] + G22 * sg[2][q]);
        if (incr)
          v += (sc[3][q] * sT[q] * JxW + sc[4][q] * (b0 * sg[0][q] + b1 * sg[1][q] + b2 * sg[2][q])) * pu;
      }
      s += pt * v + gt[0] * f0 + gt[1] * f1 + gt[2] * f2;
    }
    Ac[e] = s;
  }
}

// adds to the element matrices of the listed cells their boundary faces'
// matrices: sum over the face's Gauss points of (alpha + 4 eps sigma T^3) ds
// phi_t phi_u for the faces whose boundary id conv_bits / rad_bits selects
// (heat_diffuse_operator.cpp:1088-1129; T read plain at the face DoFs)
template <int P>
__global__ void elem_face_matrix_kernel(const KP<double> p, const long *cells, const int8_t *cell_fids,
                                        const double *cellvert, int conv_bits, double alpha, int rad_bits,
                                        double es, double *A)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  const Tables<double> &T = tab<double>(P);
  __shared__ double cq[n2];
  const long cell = cells[blockIdx.x];
  double *Ac = A + (long)blockIdx.x * n3 * n3;
  for (int f = 0; f < 6; ++f) {
    const int id = cell_fids[cell * 6 + f];
    if (id < 0) continue;  // block-uniform
    const int conv = (conv_bits >> id) & 1, rad = (rad_bits >> id) & 1;
    if (!conv && !rad) continue;
    const int d = f >> 1, s = f & 1, t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
    auto local = [&](int a, int b) {
      int loc[3];
      loc[d] = s ? P : 0;
      loc[t0] = a;
      loc[t1] = b;
      return (loc[2] * n + loc[1]) * n + loc[0];
    };
    __syncthreads();
    for (int q = threadIdx.x; q < n2; q += blockDim.x) {
      const int qa = q % n, qb = q / n;
      double xi[3];
      xi[d] = s ? 1.0 : 0.0;
      xi[t0] = T.x[qa];
      xi[t1] = T.x[qb];
      double Ja[3] = {0, 0, 0}, Jb[3] = {0, 0, 0};
      for (int v = 0; v < 8; ++v) {
        const int bv[3] = {v & 1, (v >> 1) & 1, (v >> 2) & 1};
        double fv[3], dfv[3];
        for (int c = 0; c < 3; ++c) {
          fv[c] = bv[c] ? xi[c] : 1.0 - xi[c];
          dfv[c] = bv[c] ? 1.0 : -1.0;
        }
        double da = dfv[t0], db = dfv[t1];
        for (int c = 0; c < 3; ++c)
          if (c != t0) da *= fv[c];
        for (int c = 0; c < 3; ++c)
          if (c != t1) db *= fv[c];
        for (int c = 0; c < 3; ++c) {
          const double x = cellvert[(cell * 8 + v) * 3 + c];
          Ja[c] += x * da;
          Jb[c] += x * db;
        }
      }
      const double cr[3] = {Ja[1] * Jb[2] - Ja[2] * Jb[1], Ja[2] * Jb[0] - Ja[0] * Jb[2],
                            Ja[0] * Jb[1] - Ja[1] * Jb[0]};
      const double ds = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) * T.w[qa] * T.w[qb];
      double Tq = 0.0;
      if (rad)
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) Tq += T.S[qa * n + a] * T.S[qb * n + b] * p.T[p.cmap[cell * n3 + local(a, b)]];
      cq[q] = ((conv ? alpha : 0.0) + (rad ? 4.0 * es * Tq * Tq * Tq : 0.0)) * ds;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n2 * n2; e += blockDim.x) {
      const int tf = e / n2, uf = e % n2;
      const int ta = tf % n, tb = tf / n, ua = uf % n, ub = uf / n;
      double sum = 0.0;
      for (int q = 0; q < n2; ++q) {
        const int qa = q % n, qb = q / n;
        sum += cq[q] * T.S[qa * n + ta] * T.S[qb * n + tb] * T.S[qa * n + ua] * T.S[qb * n + ub];
      }
      Ac[local(ta, tb) * n3 + local(ua, ub)] += sum;
    }
  }
}

// element matrices of the listed cells with the SUPG terms of the
// advection-diffusion tangent (advection_diffusion_operator.cpp:471-493): the
// matrix above plus tau_K (b.grad phi_t) (c_mass phi_u + c_vel b.grad phi_u / JxW
// - c_diff lap phi_u), lap phi_u = G : H_xi(phi_u) / JxW - lam . grad_xi phi_u
// (second reference derivatives of the basis: D2 = Dc D, the collocation
// derivative of its derivative at the Gauss points, as the cell kernel takes them)
template <int P>
__global__ void elem_matrix_supg_kernel(const KP<double> p, const long *cells, double *A)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  const Tables<double> &T = tab<double>(P);
  __shared__ double D2[n * n];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int q = e / n, i = e % n;
    double s = 0.0;
    for (int r = 0; r < n; ++r) s += T.Dc[q * n + r] * T.D[r * n + i];
    D2[e] = s;
  }
  __syncthreads();
  const long cell = cells[blockIdx.x];
  const double *m = p.metric + cell * metric_stride(n);
  const double *vb = p.velb ? p.velb + cell * velb_stride(n) : nullptr;  // null: no velocity
  const double *lm = p.lam ? p.lam + cell * 3 * n3 : nullptr;
  const double tau = p.tau[cell];
  double *Ac = A + (long)blockIdx.x * n3 * n3;
  for (int e = threadIdx.x; e < n3 * n3; e += blockDim.x) {
    const int t = e / n3, u = e % n3;
    const int tc[3] = {t % n, (t / n) % n, t / n2}, uc[3] = {u % n, (u / n) % n, u / n2};
    double s = 0.0;
    for (int q = 0; q < n3; ++q) {
      const int qc[3] = {q % n, (q / n) % n, q / n2};
      double st[3], dt[3], su[3], du[3], d2u[3];
      for (int d = 0; d < 3; ++d) {
        st[d] = T.S[qc[d] * n + tc[d]];
        dt[d] = T.D[qc[d] * n + tc[d]];
        su[d] = T.S[qc[d] * n + uc[d]];
        du[d] = T.D[qc[d] * n + uc[d]];
        d2u[d] = D2[qc[d] * n + uc[d]];
      }
      const double pt = st[0] * st[1] * st[2], pu = su[0] * su[1] * su[2];
      const double gt[3] = {dt[0] * st[1] * st[2], st[0] * dt[1] * st[2], st[0] * st[1] * dt[2]};
      const double gu[3] = {du[0] * su[1] * su[2], su[0] * du[1] * su[2], su[0] * su[1] * du[2]};
      const double JxW = m[q], G00 = m[n3 + q], G01 = m[2 * n3 + q], G02 = m[3 * n3 + q],
                   G11 = m[4 * n3 + q], G12 = m[5 * n3 + q], G22 = m[6 * n3 + q];
      const double b0 = vb ? vb[q] : 0.0, b1 = vb ? vb[n3 + q] : 0.0, b2 = vb ? vb[2 * n3 + q] : 0.0;
      const double adv_u = b0 * gu[0] + b1 * gu[1] + b2 * gu[2], adv_t = b0 * gt[0] + b1 * gt[1] + b2 * gt[2];
      double v = p.c_mass * JxW * pt * pu + pt * p.c_vel * adv_u;
      const double f0 = G00 * gu[0] + G01 * gu[1] + G02 * gu[2];
      const double f1 = G01 * gu[0] + G11 * gu[1] + G12 * gu[2];
      const double f2 = G02 * gu[0] + G12 * gu[1] + G22 * gu[2];
      v += p.c_diff * (gt[0] * f0 + gt[1] * f1 + gt[2] * f2);
      double r = p.c_mass * pu + p.c_vel * adv_u / JxW;
      if (p.supg_lap) {
        const double hxx = d2u[0] * su[1] * su[2], hyy = su[0] * d2u[1] * su[2], hzz = su[0] * su[1] * d2u[2];
        const double hxy = du[0] * du[1] * su[2], hxz = du[0] * su[1] * du[2], hyz = su[0] * du[1] * du[2];
        double lap = (G00 * hxx + G11 * hyy + G22 * hzz + 2.0 * (G01 * hxy + G02 * hxz + G12 * hyz)) / JxW;
        if (lm) lap -= lm[q] * gu[0] + lm[n3 + q] * gu[1] + lm[2 * n3 + q] * gu[2];
        r -= p.c_diff * lap;
      }
      v += tau * adv_t * r;
      s += v;
    }
    Ac[e] = s;
  }
}

// one warp per task (constrained-cell slot, target DoF): w^T A w, with w_t the
// weight of the target in local DoF t's entries (itself, or its constraint)
template <int P>
__global__ void __launch_bounds__(128) cell_task_kernel(long n_tasks, const int *task_cc, const long *task_tgt,
                                                        const long *ccells, const int *cmap, const int *cons_of,
                                                        const long *cptr, const long *cmast, const double *cw,
                                                        const double *A, double *val)
{
  constexpr int n = P + 1, n3 = n * n * n;
  __shared__ double ws[4][n3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long task = (long)blockIdx.x * 4 + warp;
  if (task >= n_tasks) return;  // warp-uniform
  const int cc = task_cc[task];
  const long target = task_tgt[task];
  const long cell = ccells[cc];
  double *w = ws[warp];
  for (int t = lane; t < n3; t += 32) {
    const long g = cmap[cell * n3 + t];
    const int ci = cons_of[g];
    double x = 0.0;
    if (ci < 0) {
      x = (g == target) ? 1.0 : 0.0;
    } else {
      for (long e = cptr[ci]; e < cptr[ci + 1]; ++e)
        if (cmast[e] == target) x += cw[e];
    }
    w[t] = x;
  }
  __syncwarp();
  const double *Ac = A + (long)cc * n3 * n3;
  double s = 0.0;
  for (int t = lane; t < n3; t += 32) {
    if (w[t] == 0.0) continue;
    double r = 0.0;
    for (int u = 0; u < n3; ++u) r += Ac[t * n3 + u] * w[u];
    s += w[t] * r;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) val[task] = s;
}

// per target DoF: add its tasks' values in the fixed task order
__global__ void task_fold_kernel(long n_targets, const long *tgt, const long *tptr, const double *val,
                                 double *diag)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_targets) return;
  double s = 0.0;
  for (long e = tptr[t]; e < tptr[t + 1]; ++e) s += val[e];
  diag[tgt[t]] += s;
}

// ------------------------------------------------------------------ host

namespace {

template <typename T>
T *upload(const std::vector<T> &v, size_t &bytes)
{
  if (v.empty()) return nullptr;
  T *d = dev_alloc<T>(v.size(), bytes);
  MPDG_CUDA(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return d;
}

}  // namespace

void build_mapped_mesh(Mesh &m, const mpdg_mapped_mesh_desc &d)
{
  upload_tables();
  const int p = d.degree, n = p + 1, n3 = n * n * n;
  const long E = d.n_cells, N = d.n_dofs;
  m.mapped = true;
  m.degree = p;
  m.n = n;
  m.N = m.N_own = N;
  m.n_cells = E;
  m.uniform = false;
  for (long e = 0; e < E * n3; ++e)
    if (d.cell_dofs[e] < 0 || d.cell_dofs[e] >= N) throw Error{MPDG_ERR_ARG, "cell DoF index out of range"};
  if (N >= (1L << 31)) throw Error{MPDG_ERR_SIZE, "mapped meshes hold fewer than 2^31 DoFs"};
  // constraints: validate, per-DoF index, transposed (per master) lists
  std::vector<int> cons_of(N, -1);
  std::vector<long> cdof, cptr(1, 0), cmast;
  std::vector<double> cw;
  for (long c = 0; c < d.n_constraints; ++c) {
    const long g = d.constrained_dofs[c];
    if (g < 0 || g >= N) throw Error{MPDG_ERR_ARG, "constrained DoF out of range"};
    if (cons_of[g] >= 0) throw Error{MPDG_ERR_ARG, "a DoF is constrained twice"};
    cons_of[g] = (int)c;
    cdof.push_back(g);
    for (long e = d.constraint_offsets[c]; e < d.constraint_offsets[c + 1]; ++e) {
      const long mm = d.constraint_masters[e];
      if (mm < 0 || mm >= N) throw Error{MPDG_ERR_ARG, "constraint master out of range"};
      cmast.push_back(mm);
      cw.push_back(d.constraint_weights[e]);
    }
    cptr.push_back((long)cmast.size());
  }
  for (long mm : cmast)
    if (cons_of[mm] >= 0) throw Error{MPDG_ERR_ARG, "constraint masters must be unconstrained (close the chains)"};
  std::vector<long> mdof, mptr(1, 0), mcons;
  std::vector<double> mw;
  {
    std::vector<std::vector<std::pair<long, double>>> by_master;
    std::vector<long> master_slot(N, -1);
    for (long c = 0; c < (long)cdof.size(); ++c)
      for (long e = cptr[c]; e < cptr[c + 1]; ++e) {
        const long mm = cmast[e];
        if (master_slot[mm] < 0) {
          master_slot[mm] = (long)mdof.size();
          mdof.push_back(mm);
          by_master.emplace_back();
        }
        by_master[master_slot[mm]].push_back({cdof[c], cw[e]});
      }
    for (auto &lst : by_master) {
      for (auto &pr : lst) {
        mcons.push_back(pr.first);
        mw.push_back(pr.second);
      }
      mptr.push_back((long)mcons.size());
    }
  }
  // greedy colouring: a cell takes the lowest colour none of its DoFs carries yet
  std::vector<uint64_t> used(N, 0);
  std::vector<int> colour_of(E);
  int n_col = 0;
  for (long e = 0; e < E; ++e) {
    uint64_t forbidden = 0;
    for (int t = 0; t < n3; ++t) forbidden |= used[d.cell_dofs[e * n3 + t]];
    if (~forbidden == 0) throw Error{MPDG_ERR_UNSUPPORTED, "mapped mesh needs more than 64 cell colours"};
    int c = 0;
    while ((forbidden >> c) & 1u) ++c;
    colour_of[e] = c;
    n_col = std::max(n_col, c + 1);
    for (int t = 0; t < n3; ++t) used[d.cell_dofs[e * n3 + t]] |= (uint64_t)1 << c;
  }
  m.mcol.assign(n_col, Colour{});
  for (long e = 0; e < E; ++e) m.mcol[colour_of[e]].count++;
  long first = 0;
  for (auto &C : m.mcol) {
    C.first = first;
    first += C.count;
    // no lattice: the kernels' cell position decode is unused (the map gives the DoFs)
    C.cn[0] = C.cn[1] = C.cn[2] = 1;
    C.par[0] = C.par[1] = C.par[2] = 0;
  }
  std::vector<long> next(n_col);
  for (int c = 0; c < n_col; ++c) next[c] = m.mcol[c].first;
  std::vector<int> cmap((size_t)E * n3);
  std::vector<double> cvert((size_t)E * 24);
  std::vector<uint8_t> flags(E, 0);
  std::vector<uint32_t> cmask(4 * (size_t)E, 0u);  // Dirichlet local DoFs (bit t), for the warp kernel
  // first touch: the cell of the lowest colour among a DoF's cells stores it
  // (colours launch in order and no two cells of a colour share a DoF)
  std::vector<uint32_t> cfirst(4 * (size_t)E, 0u);
  for (long e = 0; e < E; ++e) {
    const long slot = next[colour_of[e]]++;
    uint8_t f = 0;
    for (int t = 0; t < n3; ++t) {
      const long g = d.cell_dofs[e * n3 + t];
      cmap[slot * n3 + t] = (int)g;
      if (colour_of[e] == __builtin_ctzll(used[g])) cfirst[4 * slot + t / 32] |= 1u << (t % 32);
      if (d.dirichlet_mask && d.dirichlet_mask[g]) {
        f |= 1;
        cmask[4 * slot + t / 32] |= 1u << (t % 32);
      }
      if (cons_of[g] >= 0) f |= 2;
    }
    flags[slot] = f;
    for (int k = 0; k < 24; ++k) cvert[slot * 24 + k] = d.cell_vertices[e * 24 + k];
    if (f & 2) m.ccells.push_back(slot);
  }
  std::sort(m.ccells.begin(), m.ccells.end());
  // the lattice colours are unused on a mapped mesh; one colour covering all
  // cells keeps the kernels that decode lattice positions (for fields they do
  // not read here) within range
  for (int c = 0; c < 8; ++c) {
    m.colour[c] = Colour{};
    m.colour[c].cn[0] = m.colour[c].cn[1] = m.colour[c].cn[2] = 1;
    m.colour[c].first = (c == 0) ? 0 : E;
    m.colour[c].count = (c == 0) ? E : 0;
  }
  size_t &B = m.device_bytes;
  m.d_cmap = upload(cmap, B);
  m.d_cell_first = upload(cfirst, B);
  // boundary faces: greedy face colours (no two faces of a colour share a DoF)
  if (d.face_ids) {
    std::vector<uint64_t> fused(N, 0);
    std::vector<std::vector<std::array<int, 3>>> by_colour;  // (slot, local face, id)
    std::vector<long> slot_of(E);
    {
      std::vector<long> nxt(n_col);
      for (int c = 0; c < n_col; ++c) nxt[c] = m.mcol[c].first;
      for (long e = 0; e < E; ++e) slot_of[e] = nxt[colour_of[e]]++;
    }
    const int P = d.degree;
    for (long e = 0; e < E; ++e)
      for (int f = 0; f < 6; ++f) {
        const int id = d.face_ids[e * 6 + f];
        if (id < 0) continue;
        if (id > 5) throw Error{MPDG_ERR_ARG, "face ids are -1 or 0..5"};
        const int fd = f >> 1, fs = f & 1, t0 = (fd == 0) ? 1 : 0, t1 = (fd == 2) ? 1 : 2;
        std::vector<long> fg;
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            int loc[3];
            loc[fd] = fs ? P : 0;
            loc[t0] = a;
            loc[t1] = b;
            const long g = d.cell_dofs[e * n3 + (loc[2] * n + loc[1]) * n + loc[0]];
            fg.push_back(g);
          }
        uint64_t forbidden = 0;
        for (long g : fg) forbidden |= fused[g];
        if (~forbidden == 0) throw Error{MPDG_ERR_UNSUPPORTED, "mapped mesh needs more than 64 face colours"};
        int c = 0;
        while ((forbidden >> c) & 1u) ++c;
        for (long g : fg) fused[g] |= (uint64_t)1 << c;
        if ((int)by_colour.size() <= c) by_colour.resize(c + 1);
        by_colour[c].push_back({(int)slot_of[e], f, id});
      }
    std::vector<int8_t> slot_fids((size_t)E * 6);
    for (long e = 0; e < E; ++e)
      for (int f = 0; f < 6; ++f) slot_fids[(size_t)slot_of[e] * 6 + f] = d.face_ids[e * 6 + f];
    m.d_cell_fids = upload(slot_fids, B);
    std::vector<int> fcell;
    std::vector<int8_t> ff, fid;
    m.mface_first.assign(1, 0);
    for (auto &lst : by_colour) {
      for (auto &x : lst) {
        fcell.push_back(x[0]);
        ff.push_back((int8_t)x[1]);
        fid.push_back((int8_t)x[2]);
      }
      m.mface_first.push_back((long)fcell.size());
    }
    if (!fcell.empty()) {
      m.d_mface_cell = upload(fcell, B);
      m.d_mface_f = upload(ff, B);
      m.d_mface_id = upload(fid, B);
    }
  }
  m.all_dofs_touched = std::all_of(used.begin(), used.end(), [](uint64_t u) { return u != 0; });
  m.d_cellvert = upload(cvert, B);
  m.d_cell_flags = upload(flags, B);
  m.d_ccells = upload(m.ccells, B);
  m.n_cons = (long)cdof.size();
  m.n_masters = (long)mdof.size();
  m.d_cons_dof = upload(cdof, B);
  m.d_cons_ptr = upload(cptr, B);
  m.d_cons_mast = upload(cmast, B);
  m.d_cons_w = upload(cw, B);
  m.d_mast_dof = upload(mdof, B);
  m.d_mast_ptr = upload(mptr, B);
  m.d_mast_cons = upload(mcons, B);
  m.d_mast_w = upload(mw, B);
  m.d_cons_of = upload(cons_of, B);
  // masks: Dirichlet; Dirichlet or constrained; constrained
  std::vector<uint8_t> dir(N, 0), dc(N, 0), cc(N, 0);
  bool any_dir = false;
  for (long g = 0; g < N; ++g) {
    dir[g] = d.dirichlet_mask ? d.dirichlet_mask[g] : 0;
    any_dir = any_dir || dir[g];
    cc[g] = cons_of[g] >= 0;
    dc[g] = dir[g] || cc[g];
  }
  m.has_dirichlet = any_dir;
  if (any_dir) {
    m.d_dmask = upload(dir, B);
    m.d_cell_mask = upload(cmask, B);
  }
  m.d_tmask_dir = upload(dc, B);
  m.d_tmask_hang = upload(cc, B);
  // geometry: JxW and G per (cell, q) from each cell's corners
  double xw[2 * kMaxN], xq[kMaxN], wq[kMaxN];
  gauss(n, xq, wq);
  for (int q = 0; q < n; ++q) {
    xw[q] = xq[q];
    xw[kMaxN + q] = wq[q];
  }
  double *d_xw = nullptr;
  MPDG_CUDA(tracked_malloc(&d_xw, sizeof(xw)));
  MPDG_CUDA(cudaMemcpy(d_xw, xw, sizeof(xw), cudaMemcpyHostToDevice));
  m.d_metric64 = dev_alloc<double>((size_t)E * metric_stride(n), B);
  MPDG_CUDA(cudaMemset(m.d_metric64, 0, sizeof(double) * E * metric_stride(n)));
  metric_kernel<<<grid_for(E * n3, 256), 256>>>(nullptr, 0, 0, E, p, nullptr, m.d_cellvert, m.d_metric64,
                                                nullptr, d_xw, d_xw + kMaxN);
  MPDG_LAUNCHED();
  MPDG_CUDA(cudaDeviceSynchronize());
  cudaFree(d_xw);
}

template <typename Real>
void mapped_condense(Op &op, Real *dst)
{
  Mesh &m = *op.mesh;
  if (!m.n_cons) return;
  const bool mask = op.use_dirichlet && m.has_dirichlet;
  cons_condense_kernel<Real><<<grid_for(m.n_masters, 256), 256, 0, op.stream>>>(
      dst, m.n_masters, m.d_mast_dof, m.d_mast_ptr, m.d_mast_cons, m.d_mast_w, mask ? m.d_dmask : nullptr);
  MPDG_LAUNCHED();
  cons_zero_kernel<Real><<<grid_for(m.n_cons, 256), 256, 0, op.stream>>>(dst, m.n_cons, m.d_cons_dof);
  MPDG_LAUNCHED();
}

// the Dirichlet-and-constraint handling of a mapped mesh around the cell loop
template <typename Real>
void launch_mapped_apply(Op &op, Real *dst, const Real *src)
{
  Mesh &m = *op.mesh;
  const long N = m.N;
  const bool mask = op.use_dirichlet && m.has_dirichlet;
  const Real *in = src;
  if (m.n_cons) {
    const size_t bytes = sizeof(Real) * (size_t)N;
    if (op.io_tmp_bytes < bytes) {
      MPDG_CUDA(cudaStreamSynchronize(op.stream));
      if (op.io_tmp) cudaFree(op.io_tmp);
      op.io_tmp = nullptr;
      op.io_tmp_bytes = 0;
      MPDG_CUDA(tracked_malloc(&op.io_tmp, bytes));
      op.io_tmp_bytes = bytes;
    }
    Real *tmp = static_cast<Real *>(op.io_tmp);
    MPDG_CUDA(cudaMemcpyAsync(tmp, src, bytes, cudaMemcpyDeviceToDevice, op.stream));
    cons_distribute_kernel<Real><<<grid_for(m.n_cons, 256), 256, 0, op.stream>>>(
        src, tmp, m.n_cons, m.d_cons_dof, m.d_cons_ptr, m.d_cons_mast, m.d_cons_w, mask ? m.d_dmask : nullptr);
    MPDG_LAUNCHED();
    in = tmp;
  }
  KP<Real> k = base_params<Real>(op);
  k.src = in;
  k.dst = dst;
  if (sizeof(Real) == 4) {
    ensure_metric32(m, op.stream);
    k.metric = (const Real *)(const void *)m.d_metric32;
    if (op.d.vel_kind != MPDG_VEL_NONE && !op.d_velb32)
      throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
  }
  const bool kt = uses_kT(op);
  if (kt && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  check_law_fields(op, k);
  // the block kernels add into dst; the warp kernel stores each DoF's first
  // touch, so dst needs clearing only where no cell touches a DoF
  const bool warp_path = !supg(op) && !kt && !uses_law(op);
  if (!warp_path || !m.all_dofs_touched || !m.d_cell_first)
    MPDG_CUDA(cudaMemsetAsync(dst, 0, sizeof(Real) * N, op.stream));
  if (supg(op)) {
    // SUPG: the block kernel with the stabilisation flux through the map
    if constexpr (sizeof(Real) == 4) {
      if (!op.d_tau32) throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
    }
    dispatch_degree<Real, MODE_SUPG, false>(op, k);
  } else if (!kt && !uses_law(op)) {
    // constant coefficients: the warp kernel on the merged coefficient stream
    ensure_coef(op, sizeof(Real) == 4);
    if constexpr (sizeof(Real) == 8) k.metric = op.d_coef64;
    else k.metric = op.d_coef32;
    warp_apply_degree<Real, GEOM_GENERAL>(op, k);
  } else if (kt) {
    dispatch_degree<Real, MODE_LINEAR, true>(op, k);
  } else {
    dispatch_degree<Real, MODE_LINEAR, false>(op, k);
  }
  launch_robin<Real>(op, dst, in, ROBIN_APPLY);  // boundary faces selected by the cells' ids
  mapped_condense<Real>(op, dst);
}

namespace {
// diagonal contributions w^T A_K w of the cells `cells` (device copy d_cells)
// through their element matrices: the constrained cells of a mapped mesh, or
// with `supg` every cell (SUPG element matrices)
template <int P>
void mapped_element_diagonal(Op &op, double *diag, const std::vector<long> &cells, const long *d_cells, bool supg)
{
  Mesh &m = *op.mesh;
  constexpr int n = P + 1, n3 = n * n * n;
  const long ncc = (long)cells.size();
  if (ncc == 0) return;
  // tasks: every DoF (target) of every constrained cell, sorted by target
  std::vector<int> hmap((size_t)ncc * n3);
  {
    std::vector<int> all((size_t)m.n_cells * n3);
    MPDG_CUDA(cudaMemcpy(all.data(), m.d_cmap, sizeof(int) * all.size(), cudaMemcpyDeviceToHost));
    for (long c = 0; c < ncc; ++c)
      for (int t = 0; t < n3; ++t) hmap[(size_t)c * n3 + t] = all[(size_t)cells[c] * n3 + t];
  }
  std::vector<int> cons_of(m.N);
  MPDG_CUDA(cudaMemcpy(cons_of.data(), m.d_cons_of, sizeof(int) * m.N, cudaMemcpyDeviceToHost));
  std::vector<long> cptr(m.n_cons + 1), cmast;
  MPDG_CUDA(cudaMemcpy(cptr.data(), m.d_cons_ptr, sizeof(long) * cptr.size(), cudaMemcpyDeviceToHost));
  cmast.resize(cptr.back());
  if (!cmast.empty())
    MPDG_CUDA(cudaMemcpy(cmast.data(), m.d_cons_mast, sizeof(long) * cmast.size(), cudaMemcpyDeviceToHost));
  std::vector<std::pair<long, int>> tasks;  // (target, cell slot)
  for (long c = 0; c < ncc; ++c) {
    std::vector<long> tg;
    for (int t = 0; t < n3; ++t) {
      const long g = hmap[(size_t)c * n3 + t];
      if (cons_of[g] < 0) tg.push_back(g);
      else
        for (long e = cptr[cons_of[g]]; e < cptr[cons_of[g] + 1]; ++e) tg.push_back(cmast[e]);
    }
    std::sort(tg.begin(), tg.end());
    tg.erase(std::unique(tg.begin(), tg.end()), tg.end());
    for (long g : tg) tasks.push_back({g, (int)c});
  }
  std::stable_sort(tasks.begin(), tasks.end(), [](const std::pair<long, int> &a, const std::pair<long, int> &b) {
    return a.first < b.first;
  });
  std::vector<int> task_cc(tasks.size());
  std::vector<long> task_tgt(tasks.size()), tgt, tptr(1, 0);
  for (size_t i = 0; i < tasks.size(); ++i) {
    task_tgt[i] = tasks[i].first;
    task_cc[i] = tasks[i].second;
    if (tgt.empty() || tgt.back() != tasks[i].first) {
      if (!tgt.empty()) tptr.push_back((long)i);
      tgt.push_back(tasks[i].first);
    }
  }
  tptr.push_back((long)tasks.size());
  // device scratch: element matrices, task arrays, task values
  size_t scratch = 0;
  double *A = dev_alloc<double>((size_t)ncc * n3 * n3, scratch);
  double *val = nullptr;
  int *d_task_cc = nullptr;
  long *d_task_tgt = nullptr, *d_tgt = nullptr, *d_tptr = nullptr;
  try {
    val = dev_alloc<double>(tasks.size(), scratch);
    d_task_cc = upload(task_cc, scratch);
    d_task_tgt = upload(task_tgt, scratch);
    d_tgt = upload(tgt, scratch);
    d_tptr = upload(tptr, scratch);
    KP<double> k = base_params<double>(op);
    if (supg) elem_matrix_supg_kernel<P><<<(unsigned)ncc, 256, 0, op.stream>>>(k, d_cells, A);
    else if (uses_kT(op)) elem_matrix_field_kernel<P><<<(unsigned)ncc, 256, 0, op.stream>>>(k, d_cells, A);
    else elem_matrix_kernel<P><<<(unsigned)ncc, 256, 0, op.stream>>>(k, d_cells, A);
    MPDG_LAUNCHED();
    const mpdg_op_desc &D = op.d;
    const int conv_bits = (D.kind == MPDG_OP_HEAT && D.robin_alpha != 0.0) ? D.robin_faces : 0;
    const int rad_bits = (D.kind == MPDG_OP_HEAT && D.rad_emissivity != 0.0) ? D.rad_faces : 0;
    if (!supg && m.d_cell_fids && (conv_bits || rad_bits)) {
      if (rad_bits && !op.T64) throw Error{MPDG_ERR_ARG, "radiative faces need the temperature field"};
      elem_face_matrix_kernel<P><<<(unsigned)ncc, 128, 0, op.stream>>>(
          k, d_cells, m.d_cell_fids, m.d_cellvert, conv_bits, D.robin_alpha, rad_bits,
          D.rad_emissivity * 5.670374419e-8, A);
      MPDG_LAUNCHED();
    }
    const long nt = (long)tasks.size();
    cell_task_kernel<P><<<(unsigned)((nt + 3) / 4), 128, 0, op.stream>>>(
        nt, d_task_cc, d_task_tgt, d_cells, m.d_cmap, m.d_cons_of, m.d_cons_ptr, m.d_cons_mast, m.d_cons_w, A,
        val);
    MPDG_LAUNCHED();
    task_fold_kernel<<<grid_for((long)tgt.size(), 256), 256, 0, op.stream>>>((long)tgt.size(), d_tgt, d_tptr, val,
                                                                              diag);
    MPDG_LAUNCHED();
    MPDG_CUDA(cudaStreamSynchronize(op.stream));
  } catch (...) {
    cudaStreamSynchronize(op.stream);
    for (void *q : {(void *)A, (void *)val, (void *)d_task_cc, (void *)d_task_tgt, (void *)d_tgt, (void *)d_tptr})
      if (q) cudaFree(q);
    throw;
  }
  for (void *q : {(void *)A, (void *)val, (void *)d_task_cc, (void *)d_task_tgt, (void *)d_tgt, (void *)d_tptr})
    if (q) cudaFree(q);
}
}  // namespace

// diagonal of sum_K C_K^T A_K C_K: separable diagonals of the unconstrained
// cells, element-matrix quadratic forms of the constrained ones; 1 at the
// constrained DoFs and (with the Dirichlet set selected) at the Dirichlet DoFs
void launch_mapped_diagonal(Op &op, double *diag)
{
  Mesh &m = *op.mesh;
  KP<double> k = base_params<double>(op);
  k.dst = diag;
  k.skip_constrained = 1;
  const bool kt = uses_kT(op);
  if (kt && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  check_law_fields(op, k);
  MPDG_CUDA(cudaMemsetAsync(diag, 0, sizeof(double) * m.N, op.stream));
  if (supg(op)) {
    // SUPG: the element matrices of every cell, in chunks of cells that bound
    // the scratch (the diagonal is built once per operator)
    if (!op.d_tau64) throw Error{MPDG_ERR_ARG, "SUPG diagonal: tau missing"};
    const long chunk = 16384;
    for (long c0 = 0; c0 < m.n_cells; c0 += chunk) {
      std::vector<long> cells;
      for (long c = c0; c < std::min(m.n_cells, c0 + chunk); ++c) cells.push_back(c);
      size_t scratch = 0;
      long *d_cells = upload(cells, scratch);
      try {
        switch (m.degree) {
          case 1: mapped_element_diagonal<1>(op, diag, cells, d_cells, true); break;
          case 2: mapped_element_diagonal<2>(op, diag, cells, d_cells, true); break;
          case 3: mapped_element_diagonal<3>(op, diag, cells, d_cells, true); break;
          case 4: mapped_element_diagonal<4>(op, diag, cells, d_cells, true); break;
          default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
        }
      } catch (...) {
        cudaStreamSynchronize(op.stream);
        cudaFree(d_cells);
        throw;
      }
      MPDG_CUDA(cudaStreamSynchronize(op.stream));
      cudaFree(d_cells);
    }
  } else {
    switch (m.degree) {
      case 1:
        kt ? run_diag<1, true>(op, k) : run_diag<1, false>(op, k);
        mapped_element_diagonal<1>(op, diag, m.ccells, m.d_ccells, false);
        break;
      case 2:
        kt ? run_diag<2, true>(op, k) : run_diag<2, false>(op, k);
        mapped_element_diagonal<2>(op, diag, m.ccells, m.d_ccells, false);
        break;
      case 3:
        kt ? run_diag<3, true>(op, k) : run_diag<3, false>(op, k);
        mapped_element_diagonal<3>(op, diag, m.ccells, m.d_ccells, false);
        break;
      case 4:
        kt ? run_diag<4, true>(op, k) : run_diag<4, false>(op, k);
        mapped_element_diagonal<4>(op, diag, m.ccells, m.d_ccells, false);
        break;
      default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
    }
  }
  launch_robin<double>(op, diag, nullptr, ROBIN_DIAGONAL);
  const uint8_t *tm = op.use_dirichlet ? m.d_tmask_dir : m.d_tmask_hang;
  set_masked_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, tm, 1.0);
  MPDG_LAUNCHED();
}
