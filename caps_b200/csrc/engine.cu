// Host side of the device engine: the C ABI of include/caps_gpu.h, force-field upload, cell and list geometry, and the
// kernel sequence of one force evaluation (Evaluator::compute, core/src/field.cpp:1249-2539).
#include "engine.h"
#include "caps_gpu_diag.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>


namespace capsb {

// ---------------------------------------------------------------------------------------------------------------

namespace {

// Ewald coefficient by bisection of erfc(beta rc) = rtol (core/src/kspace.cpp:35-43).
double ewald_beta(double cutoff, double rtol) {
  double lo = 0, hi = 20.0 / cutoff;
  for (int it = 0; it < 100; ++it) {
    const double mid = 0.5 * (lo + hi);
    (std::erfc(mid * cutoff) > rtol ? lo : hi) = mid;
  }
  return 0.5 * (lo + hi);
}

// smallest n' >= n with prime factors 2, 3, 5, 7 (caps_kspace.f90:23-36)
int good_size(int n) {
  int m = std::max(n, 1);
  for (;;) {
    int k = m;
    while (k % 2 == 0) k /= 2;
    while (k % 3 == 0) k /= 3;
    while (k % 5 == 0) k /= 5;
    while (k % 7 == 0) k /= 7;
    if (k == 1) return m;
    ++m;
  }
}

double erfc_as_host(double x, double& ex2) {   // Abramowitz & Stegun 7.1.26 (field.cpp:585-591), used for the DSF constants
  const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741, A4 = -1.453152027, A5 = 1.061405429;
  ex2 = std::exp(-x * x);
  const double t = 1.0 / (1.0 + P * x);
  return t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ex2;
}

// |b(m)|^2 of the Euler exponential spline (caps_kspace.f90:601-620), from the order-p weights at w = 0
void bspline_moduli(int k, int p, std::vector<double>& bsp) {
  std::vector<double> th(size_t(p), 0.0);
  // bspline(0, p): the recursion of caps_kspace.f90:568-598 at w = 0
  const double w = 0;
  th[1] = w;
  th[0] = 1 - w;
  for (int kk = 3; kk <= p - 1; ++kk) {
    const double div = 1.0 / (kk - 1);
    th[size_t(kk - 1)] = div * w * th[size_t(kk - 2)];
    for (int j = 1; j <= kk - 2; ++j) th[size_t(kk - j - 1)] = div * ((w + j) * th[size_t(kk - j - 2)] + (kk - j - w) * th[size_t(kk - j - 1)]);
    th[0] = div * (1 - w) * th[0];
  }
  {
    const double div = 1.0 / (p - 1);
    th[size_t(p - 1)] = div * w * th[size_t(p - 2)];
    for (int j = 1; j <= p - 2; ++j) th[size_t(p - j - 1)] = div * ((w + j) * th[size_t(p - j - 2)] + (p - j - w) * th[size_t(p - j - 1)]);
    th[0] = div * (1 - w) * th[0];
  }
  bsp.assign(size_t(k), 0.0);
  for (int m = 0; m < k; ++m) {
    double sr = 0, si = 0;
    for (int j = 0; j <= p - 2; ++j) {
      const double arg = 2 * kPi * m * j / double(k);
      sr += th[size_t(j)] * std::cos(arg);
      si += th[size_t(j)] * std::sin(arg);
    }
    bsp[size_t(m)] = sr * sr + si * si;
  }
  for (int m = 0; m < k; ++m)
    if (bsp[size_t(m)] < 1e-7) bsp[size_t(m)] = 0.5 * (bsp[size_t(((m - 1) % k + k) % k)] + bsp[size_t((m + 1) % k)]);
}

void cell_matrices(const double* c, DevCell& d) {
  for (int k = 0; k < 3; ++k) d.o[k] = c[k];
  for (int r = 0; r < 3; ++r)
    for (int col = 0; col < 3; ++col) d.h[r][col] = c[3 + 3 * col + r];
  const auto& h = d.h;
  // the inverse as caps_kspace.f90:495-511 (cell_inverse) writes it
  const double vol = h[0][0] * (h[1][1] * h[2][2] - h[2][1] * h[1][2]) - h[0][1] * (h[1][0] * h[2][2] - h[2][0] * h[1][2]) +
                     h[0][2] * (h[1][0] * h[2][1] - h[2][0] * h[1][1]);
  d.hi[0][0] = (h[1][1] * h[2][2] - h[1][2] * h[2][1]) / vol;
  d.hi[0][1] = (h[0][2] * h[2][1] - h[0][1] * h[2][2]) / vol;
  d.hi[0][2] = (h[0][1] * h[1][2] - h[0][2] * h[1][1]) / vol;
  d.hi[1][0] = (h[1][2] * h[2][0] - h[1][0] * h[2][2]) / vol;
  d.hi[1][1] = (h[0][0] * h[2][2] - h[0][2] * h[2][0]) / vol;
  d.hi[1][2] = (h[0][2] * h[1][0] - h[0][0] * h[1][2]) / vol;
  d.hi[2][0] = (h[1][0] * h[2][1] - h[1][1] * h[2][0]) / vol;
  d.hi[2][1] = (h[0][1] * h[2][0] - h[0][0] * h[2][1]) / vol;
  d.hi[2][2] = (h[0][0] * h[1][1] - h[0][1] * h[1][0]) / vol;
  d.vol = std::fabs(vol);
}

double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// radices of n for the line FFT: 4s first, then 2, 3, 5, 7 and any other prime
}  // namespace

// ---------------------------------------------------------------------------------------------------------------
Engine::Engine(const caps_gpu_ff* ff, const caps_gpu_opts* o) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw ModelError(CAPS_GPU_ENODEV, "no CUDA device: the B200 engine has no CPU fallback");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&dev_sms_, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  // the main stream (integrator, list, pack, prune, pair kernel) runs at the highest priority, PME's chain of dependent
  // launches one level below and the bonded terms at the lowest: the chain that leads to the pair kernel takes SM
  // slots first, then PME's, and the bonded blocks fill what they leave
  int prio_lo = 0, prio_hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  CK(cudaStreamDestroy(stream_));
  CK(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, prio_hi));
  CK(cudaStreamCreateWithPriority(&side_[0], cudaStreamNonBlocking, prio_lo));
  CK(cudaStreamCreateWithPriority(&side_[1], cudaStreamNonBlocking, prio_hi < prio_lo ? prio_hi + 1 : prio_lo));
  CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
  for (auto& ev : ev_join_) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaMallocHost(&h_counters_, sizeof(int) * kCntNum));
  CK(cudaMallocHost(&h_efix_, sizeof(long long) * kENumSlots));
  CK(cudaMallocHost(&h_edbl_, sizeof(double) * kENumSlots));
  opt_ = *o;
  setup_ff(ff);
  setup_options();
}

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  stepper_.reset();
  if (h_counters_) cudaFreeHost(h_counters_);
  if (h_efix_) cudaFreeHost(h_efix_);
  if (h_edbl_) cudaFreeHost(h_edbl_);
  if (stream_) cudaStreamDestroy(stream_);
  for (auto st : side_)
    if (st) cudaStreamDestroy(st);
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  for (auto ev : ev_join_)
    if (ev) cudaEventDestroy(ev);
}

void Engine::setup_ff(const caps_gpu_ff* ff) {
  n_ = ff->natoms;
  nt_ = ff->ntypes;
  if (n_ < 1 || nt_ < 1) throw ModelError(CAPS_GPU_EINVAL, "the force field needs atoms and types");
  if (nt_ > 63) throw ModelError(CAPS_GPU_EINVAL, "at most 63 atom types on the device path");
  h_type_.assign(ff->type_index, ff->type_index + n_);
  for (int t : h_type_)
    if (t < 0 || t >= nt_) throw ModelError(CAPS_GPU_EINVAL, "type index out of range");
  h_q_.assign(ff->charge, ff->charge + n_);
  h_mass_.assign(ff->mass, ff->mass + n_);
  h_eps_.assign(ff->pair_eps, ff->pair_eps + size_t(nt_) * nt_);
  h_sig_.assign(ff->pair_sigma, ff->pair_sigma + size_t(nt_) * nt_);
  // generic pair forms (field.cpp:478-487): both orders of each type pair; the pair is evaluated whatever its LJ eps
  const size_t nt2 = size_t(nt_) * nt_;
  h_form_.assign(nt2, 0);
  h_pa_.assign(nt2, 0.0), h_pb_.assign(nt2, 0.0), h_pc_.assign(nt2, 0.0), h_prc2_.assign(nt2, 0.0);
  generic_ = false;
  for (int k = 0; k < ff->npair_func; ++k) {
    const int a = ff->pair_func_ab[2 * k], b = ff->pair_func_ab[2 * k + 1];
    const double* q = ff->pair_func_p + 5 * k;
    const int form = int(q[0]);
    if (a < 0 || b < 0 || a >= nt_ || b >= nt_) throw ModelError(CAPS_GPU_EINVAL, "a pair form refers to a type out of range");
    if (!(form == 1 || form == 2 || form == 3 || (form >= 11 && form <= 14) || form == 20 || form == 31 || form == 32 || form == 40))
      throw ModelError(CAPS_GPU_EFIELD, "unknown pair form " + std::to_string(form));
    if (form == 40 && (q[1] < 0 || int(q[1]) >= ff->ntables)) throw ModelError(CAPS_GPU_EFIELD, "a tabulated pair refers to a table that is not there");
    for (const size_t tp : {size_t(a) * nt_ + b, size_t(b) * nt_ + a}) {
      h_form_[tp] = form;
      h_pa_[tp] = q[1], h_pb_[tp] = q[2], h_pc_[tp] = q[3];
      h_prc2_[tp] = q[4] * q[4];
    }
    generic_ = true;
  }
  lj_inner_ = ff->lj_inner;
  lj_fsw_ = ff->lj_fsw != 0;
  // the tabulated pairs (ForceField::tables), one after another
  h_toff_.assign(1, 0);
  h_tr0dr_.clear(), h_te_.clear(), h_tf_.clear();
  for (int k = 0; k < ff->ntables; ++k) {
    const int m = ff->table_n[k];
    h_tr0dr_.push_back(ff->table_r0_dr[2 * k]);
    h_tr0dr_.push_back(ff->table_r0_dr[2 * k + 1]);
    h_te_.insert(h_te_.end(), ff->table_e + h_toff_.back(), ff->table_e + h_toff_.back() + m);
    h_tf_.insert(h_tf_.end(), ff->table_f + h_toff_.back(), ff->table_f + h_toff_.back() + m);
    h_toff_.push_back(h_toff_.back() + m);
  }
  d_toff_.upload(h_toff_, stream_);
  if (!h_tr0dr_.empty()) d_tr0dr_.upload(h_tr0dr_, stream_);
  if (!h_te_.empty()) {
    d_te_.upload(h_te_, stream_);
    d_tf_.upload(h_tf_, stream_);
  }
  type_count_.assign(size_t(nt_), 0.0);
  for (int t : h_type_) type_count_[size_t(t)] += 1;
  d_type_.upload(h_type_, stream_);
  d_q_.upload(h_q_, stream_);
  d_mass_.upload(h_mass_, stream_);
  auto check_idx = [&](const uint32_t* v, size_t cnt, const char* what) {
    for (size_t k = 0; k < cnt; ++k)
      if (v[k] >= uint32_t(n_)) throw ModelError(CAPS_GPU_EINVAL, std::string(what) + ": atom index out of range");
  };
  hb_.clear();
  hr0_.clear();
  ha_.clear();
  hth0_.clear();
  for (int k = 0; k < ff->nbonds; ++k) hb_.push_back({ff->bond_ij[2 * k], ff->bond_ij[2 * k + 1]}), hr0_.push_back(ff->bond_k_r0[2 * k + 1]);
  for (int k = 0; k < ff->nfene; ++k) hb_.push_back({ff->fene_ij[2 * k], ff->fene_ij[2 * k + 1]}), hr0_.push_back(0.0);
  for (int k = 0; k < ff->nangles; ++k)
    ha_.push_back({ff->angle_ijk[3 * k], ff->angle_ijk[3 * k + 1], ff->angle_ijk[3 * k + 2]}), hth0_.push_back(ff->angle_kt_theta0[2 * k + 1]);
  nb_ = ff->nbonds;
  if (nb_) {
    check_idx(ff->bond_ij, size_t(2) * nb_, "bonds");
    d_bond_ij_.upload(ff->bond_ij, size_t(2) * nb_, stream_);
    d_bond_kr_.upload(ff->bond_k_r0, size_t(2) * nb_, stream_);
  }
  na_ = ff->nangles;
  if (na_) {
    check_idx(ff->angle_ijk, size_t(3) * na_, "angles");
    d_angle_ijk_.upload(ff->angle_ijk, size_t(3) * na_, stream_);
    d_angle_kt_.upload(ff->angle_kt_theta0, size_t(2) * na_, stream_);
  }
  // torsion groups: consecutive terms on one quadruple (field.cpp:1875-1920)
  auto groups = [](int cnt, const uint32_t* q, std::vector<int>& g) {
    g.clear();
    for (int t = 0; t < cnt; ++t) {
      if (t == 0 || q[4 * t] != q[4 * (t - 1)] || q[4 * t + 1] != q[4 * (t - 1) + 1] || q[4 * t + 2] != q[4 * (t - 1) + 2] ||
          q[4 * t + 3] != q[4 * (t - 1) + 3])
        g.push_back(t);
    }
    g.push_back(cnt);
  };
  std::vector<int> grp;
  nd_ = ff->ndihedrals;
  if (nd_) {
    check_idx(ff->dihedral_ijkl, size_t(4) * nd_, "dihedrals");
    d_dih_ijkl_.upload(ff->dihedral_ijkl, size_t(4) * nd_, stream_);
    d_dih_vd_.upload(ff->dihedral_v_delta, size_t(2) * nd_, stream_);
    d_dih_n_.upload(ff->dihedral_n, size_t(nd_), stream_);
    groups(nd_, ff->dihedral_ijkl, grp);
    ndg_ = int(grp.size()) - 1;
    d_dih_grp_.upload(grp, stream_);
    CK(cudaStreamSynchronize(stream_));
  }
  ni_ = ff->nimpropers;
  if (ni_) {
    check_idx(ff->improper_ijkl, size_t(4) * ni_, "impropers");
    d_imp_ijkl_.upload(ff->improper_ijkl, size_t(4) * ni_, stream_);
    d_imp_vd_.upload(ff->improper_v_delta, size_t(2) * ni_, stream_);
    d_imp_n_.upload(ff->improper_n, size_t(ni_), stream_);
    groups(ni_, ff->improper_ijkl, grp);
    nig_ = int(grp.size()) - 1;
    d_imp_grp_.upload(grp, stream_);
    CK(cudaStreamSynchronize(stream_));
  }
  // 1-4 pairs and the Coulomb fraction each keeps (field.cpp:445-457)
  np14_ = ff->npairs14;
  lj14_ = ff->lj14;
  std::map<std::pair<uint32_t, uint32_t>, double> p14;
  if (np14_) {
    check_idx(ff->pair14_ij, size_t(2) * np14_, "pairs14");
    d_p14_ij_.upload(ff->pair14_ij, size_t(2) * np14_, stream_);
    p14_scaled_ = ff->pair14_lj != nullptr;
    if (p14_scaled_) d_p14_scale_.upload(ff->pair14_lj, size_t(np14_), stream_);
    for (int k = 0; k < np14_; ++k) {
      const uint32_t a = ff->pair14_ij[2 * k], b = ff->pair14_ij[2 * k + 1];
      p14[{std::min(a, b), std::max(a, b)}] = ff->pair14_coul ? ff->pair14_coul[k] : ff->coul14;
    }
  }
  // excluded partners: the CSR for the list, and (i < j, factor) pairs for the Coulomb corrections
  std::vector<uint32_t> eoff(size_t(n_) + 1, 0), elist, xij;
  std::vector<double> xf;
  for (int i = 0; i < n_; ++i) {
    const uint32_t b0 = ff->excl_offset ? ff->excl_offset[i] : 0, b1 = ff->excl_offset ? ff->excl_offset[i + 1] : 0;
    for (uint32_t p = b0; p < b1; ++p) {
      const uint32_t j = ff->excl_list[p];
      if (j >= uint32_t(n_)) throw ModelError(CAPS_GPU_EINVAL, "excluded: atom index out of range");
      if (j == uint32_t(i)) continue;
      elist.push_back(j);
      if (j > uint32_t(i)) {
        const auto it = p14.find({uint32_t(i), j});
        xij.push_back(uint32_t(i));
        xij.push_back(j);
        xf.push_back(it != p14.end() ? it->second : 0.0);
      }
    }
    eoff[size_t(i) + 1] = uint32_t(elist.size());
  }
  d_excl_off_.upload(eoff, stream_);
  d_excl_list_.upload(elist, stream_);
  nx_ = int(xf.size());
  if (nx_) {
    d_excl_ij_.upload(xij, stream_);
    d_excl_f_.upload(xf, stream_);
  }
  nfene_ = ff->nfene;
  if (nfene_) {
    check_idx(ff->fene_ij, size_t(2) * nfene_, "fene");
    d_fene_ij_.upload(ff->fene_ij, size_t(2) * nfene_, stream_);
    d_fene_p_.upload(ff->fene_k_r0_eps_sigma, size_t(4) * nfene_, stream_);
    h_fene_r0_.resize(size_t(nfene_));
    for (int k = 0; k < nfene_; ++k) h_fene_r0_[size_t(k)] = ff->fene_k_r0_eps_sigma[4 * k + 1];
  }
  lj_shift_model_ = ff->lj_shift != 0;
  model_cutoff_ = ff->model_cutoff;
  if (ff->lj_form != 0 && ff->lj_form != 1) throw ModelError(CAPS_GPU_EFIELD, "unknown pair form (0 lj12-6, 1 lj9-6)");
  lj96_ = ff->lj_form == 1;
  CK(cudaStreamSynchronize(stream_));
}

// The energy of a generic pair form at r^2 (field.cpp:1382-1396), for the cut-off shift.
static double generic_pair_energy(int form, double pa, double pb, double pc, double r2) {
  const double r = std::sqrt(r2);
  if (form == 1) return pa * std::exp(-r / pb) - pc / (r2 * r2 * r2);
  if (form == 3) return (pa + pc * r) * std::exp(-r / pb);
  if (form >= 11 && form <= 14) {   // SDK (field.cpp:1443-1448)
    static const double pw1[] = {9, 12, 12, 12}, pw2[] = {6, 4, 6, 5}, pre[] = {6.75, 2.59807621135332, 4.0, 3.20377984125109};
    const int k = form - 11;
    const double sr2 = pb * pb / r2, sm = std::pow(sr2, pw1[k] / 2), sn = std::pow(sr2, pw2[k] / 2), c = pre[k] * pa;
    return c * (sm - sn);
  }
  const double e1 = std::exp(-pb * (r - pc));
  return pa * (e1 * e1 - 2 * e1);
}

void Engine::setup_options() {
  rc_ = model_cutoff_ > 0 ? model_cutoff_ : opt_.cutoff;
  skin_ = opt_.skin;
  if (!(rc_ > 0) || skin_ < 0) throw ModelError(CAPS_GPU_EINVAL, "cut-off must be positive and skin non-negative");
  // a force field with generic pair forms runs the FP64 path, as the reference's mixed path falls back to its FP64
  // pair loop for them (field.cpp:848)
  mixed_ = opt_.precision == 0 && !generic_ && !lj_fsw_;
  tail_ = opt_.tail != 0 && !lj_shift_model_ && !lj_fsw_;   // CHARMM: switched to zero at the cut-off, no tail (field.cpp:440-443)
  shifted_ = !tail_;
  coul_ = opt_.coulomb != 0;
  pme_ = coul_ && opt_.electrostatics == 1;
  order_ = opt_.pme_order;
  if (pme_ && (order_ < 3 || order_ > kMaxOrder)) throw ModelError(CAPS_GPU_EINVAL, "PME order must be 3..8");
  if (lj_fsw_ && (lj_inner_ <= 0 || lj_inner_ >= rc_)) throw ModelError(CAPS_GPU_EFIELD, "the CHARMM force switch needs an inner radius below the cut-off");
  if (opt_.force_cap > 0 && mixed_) throw ModelError(CAPS_GPU_EINVAL, "a force cap runs on the FP64 path (as the reference's push-off)");
  beta_ = pme_ ? ewald_beta(rc_, opt_.ewald_rtol) : 0.0;
  const double a = opt_.dsf_alpha;
  double ex;
  erfc_rc_ = erfc_as_host(a * rc_, ex);
  dsf_e0_ = erfc_rc_ / rc_;
  dsf_f0_ = erfc_rc_ / (rc_ * rc_) + 2 * a / std::sqrt(kPi) * std::exp(-a * a * rc_ * rc_) / rc_;
  kappa_ = pme_ ? beta_ : a;
  // Ewald / DSF table G(s) = erf(kappa sqrt s)/sqrt s and h dG/ds (field.cpp:1126-1157)
  if (coul_) {
    const double smax = rc_ * rc_, kap = kappa_;
    const size_t m = std::max<size_t>(1024, size_t(std::ceil(smax * kap * kap / 0.025)));
    const double h = smax / double(m);
    const double c = 2 * kap / std::sqrt(kPi), k2 = kap * kap;
    std::vector<double> gt(2 * (m + 2), 0.0);
    for (size_t k = 0; k <= m + 1; ++k) {
      const double s = double(k) * h, x = k2 * s;
      double G, dG;
      if (x < 1) {
        G = 0, dG = 0;
        double term = 1;
        for (int nn = 0; nn < 30; ++nn) {
          G += term / (2 * nn + 1);
          dG -= term / (2 * nn + 3);
          term *= -x / (nn + 1);
        }
        G *= c;
        dG *= c * k2;
      } else {
        const double r = std::sqrt(s), e = std::erf(kap * r);
        G = e / r;
        dG = (c * std::exp(-x) - G) / (2 * s);
      }
      gt[2 * k] = G;
      gt[2 * k + 1] = h * dG;
    }
    d_gtab_.upload(gt, stream_);
    gnodes_ = int(m + 2);
    ghi_ = 1 / h;
  }
  // pair coefficient tables, the padding type last (all zero)
  const int ntab = nt_ + 1;
  std::vector<float4> tab(size_t(ntab) * ntab, make_float4(0, 0, 0, 0));
  std::vector<double4> tabd(size_t(ntab) * ntab, make_double4(0, 0, 0, 0)), l14(size_t(nt_) * nt_);
  const double rc2 = rc_ * rc_;
  for (int a0 = 0; a0 < nt_; ++a0)
    for (int b0 = 0; b0 < nt_; ++b0) {
      const double eps = h_eps_[size_t(a0) * nt_ + b0], sg = h_sig_[size_t(a0) * nt_ + b0];
      const double s6 = std::pow(sg, 6);
      // 12-6: c6 r^-6 with c6 = 4 eps s^6, and 4 eps s^12 r^-12; 9-6 (field.cpp:860-861): 3 eps s^6 and 2 eps s^9 r^-9
      const double c6 = eps > 0 ? (lj96_ ? 3 : 4) * eps * s6 : 0.0;
      const double c12 = eps > 0 ? (lj96_ ? 2 * eps * s6 * std::sqrt(s6) : 4 * eps * s6 * s6) : 0.0;
      const double qc = s6 / (rc2 * rc2 * rc2);
      const double sh = shifted_ && eps > 0 && !(lj_fsw_ && !lj96_) ? (lj96_ ? eps * (2 * qc * std::sqrt(qc) - 3 * qc) : 4 * eps * (qc * qc - qc)) : 0.0;
      tab[size_t(a0) * ntab + b0] = make_float4(float(c6), float(c12), float(sh), 0.f);
      tabd[size_t(a0) * ntab + b0] = make_double4(c6, c12, sh, 0.0);
      l14[size_t(a0) * nt_ + b0] = make_double4(eps, s6, sh, 0.0);
    }
  // generic forms: no LJ part; the shift is the form's energy at the pair's own cut-off, or at r_c, unless the tail
  // correction is on (field.cpp:1482-1492)
  // lj/gromacs: the switch coefficients for the cut-off in use (field.cpp:528-547); their constant g4 is the pair's
  // (negative) shift, and the cut-off shift is none by construction, as for the cosine-squared and tabulated forms
  std::vector<double4> tabg(size_t(ntab) * ntab, make_double4(0, 0, 0, 0)), l14g(size_t(nt_) * nt_, make_double4(0, 0, 0, 0));
  std::vector<double4> tabg2(size_t(ntab) * ntab, make_double4(0, 0, 0, 0)), l14g2(size_t(nt_) * nt_, make_double4(0, 0, 0, 0));
  for (int a0 = 0; a0 < nt_ && generic_; ++a0)
    for (int b0 = 0; b0 < nt_; ++b0) {
      const size_t tp = size_t(a0) * nt_ + b0;
      const int form = h_form_[tp];
      if (!form) continue;
      double sh = 0;
      double4 g2 = make_double4(0, 0, 0, 0);
      if (form == 20) {
        const double rc = rc_, r1 = lj_inner_;
        if (r1 <= 0 || r1 >= rc) throw ModelError(CAPS_GPU_EFIELD, "lj/gromacs needs an inner radius below the cut-off");
        const double e = h_pa_[tp], sg = h_pb_[tp], s6 = std::pow(sg, 6), s12 = s6 * s6;
        const double l1 = 48 * e * s12, l2 = 24 * e * s6, l3 = 4 * e * s12, l4 = 4 * e * s6;
        const double r6i = 1 / std::pow(rc, 6), r8i = 1 / std::pow(rc, 8), tt = rc - r1, t2i = 1 / (tt * tt), t3i = t2i / tt, t3 = tt * tt * tt;
        const double a6 = (7 * r1 - 10 * rc) * r8i * t2i, b6 = (9 * rc - 7 * r1) * r8i * t3i;
        const double a12 = (13 * r1 - 16 * rc) * r6i * r8i * t2i, b12 = (15 * rc - 13 * r1) * r6i * r8i * t3i;
        const double c6 = r6i - t3 * (6 * a6 / 3 + 6 * b6 * tt / 4), c12 = r6i * r6i - t3 * (12 * a12 / 3 + 12 * b12 * tt / 4);
        g2 = make_double4(l1 * a12 - l2 * a6, l1 * b12 - l2 * b6, -l3 * 12 * a12 / 3 + l4 * 6 * a6 / 3, -l3 * 12 * b12 / 4 + l4 * 6 * b6 / 4);
        sh = -(-l3 * c12 + l4 * c6);
      } else if (shifted_ && form != 31 && form != 32 && form != 40) {
        const double r2 = h_prc2_[tp] > 0 ? std::min(h_prc2_[tp], rc2) : rc2;
        sh = generic_pair_energy(form, h_pa_[tp], h_pb_[tp], h_pc_[tp], r2);
      }
      tabd[size_t(a0) * ntab + b0] = make_double4(0.0, 0.0, sh, double(form));
      tabg[size_t(a0) * ntab + b0] = make_double4(h_pa_[tp], h_pb_[tp], h_pc_[tp], h_prc2_[tp]);
      tabg2[size_t(a0) * ntab + b0] = g2;
      l14[tp] = make_double4(1.0, 0.0, sh, double(form));
      l14g[tp] = tabg[size_t(a0) * ntab + b0];
      l14g2[tp] = g2;
    }
  d_tabg_.upload(tabg, stream_);
  d_lj14g_.upload(l14g, stream_);
  d_tabg2_.upload(tabg2, stream_);
  d_lj14g2_.upload(l14g2, stream_);
  d_tab_.upload(tab, stream_);
  // geometric mixing (c6_ab = sqrt(c6_aa c6_bb) and the same for c12, as OPLS-style force fields give): the FP32 pair
  // kernel takes per-type factors instead of the per-pair table (12-6 only)
  comb_ = !lj96_;
  std::vector<float2> ljf(size_t(ntab), make_float2(0.f, 0.f));
  for (int a0 = 0; a0 < nt_ && comb_; ++a0) {
    const double c6a = tabd[size_t(a0) * ntab + a0].x, c12a = tabd[size_t(a0) * ntab + a0].y;
    ljf[size_t(a0)] = make_float2(float(std::sqrt(c6a)), float(std::sqrt(c12a)));
    for (int b0 = 0; b0 < nt_; ++b0) {
      const double c6b = tabd[size_t(b0) * ntab + b0].x, c12b = tabd[size_t(b0) * ntab + b0].y;
      const double c6 = tabd[size_t(a0) * ntab + b0].x, c12 = tabd[size_t(a0) * ntab + b0].y;
      if (std::fabs(c6 - std::sqrt(c6a * c6b)) > 1e-12 * std::max(c6, 1e-300) || std::fabs(c12 - std::sqrt(c12a * c12b)) > 1e-12 * std::max(c12, 1e-300))
        comb_ = false;
    }
  }
  d_ljf_.upload(ljf, stream_);
  d_tabd_.upload(tabd, stream_);
  d_lj14_.upload(l14, stream_);
  // force-cap radii (field.cpp:557-581): where |F_LJ| reaches the cap, by bisection; beyond it nothing changes
  std::vector<double4> cap(size_t(ntab) * ntab, make_double4(0, 0, 0, 0)), cap14(size_t(nt_) * nt_, make_double4(0, 0, 0, 0));
  if (opt_.force_cap > 0)
    for (int a0 = 0; a0 < nt_; ++a0)
      for (int b0 = 0; b0 < nt_; ++b0) {
        const double e = h_eps_[size_t(a0) * nt_ + b0], s6 = std::pow(h_sig_[size_t(a0) * nt_ + b0], 6);
        if (e <= 0 || h_form_[size_t(a0) * nt_ + b0] != 0) continue;   // the cap is for Lennard-Jones only
        const double sg = std::pow(s6, 1.0 / 6);
        auto force = [&](double r) {
          if (lj96_) {
            const double q = sg / r, q3 = q * q * q;
            return 18 * e / r * (q3 * q3 * q3 - q3 * q3);
          }
          const double q = s6 / std::pow(r, 6);
          return 24 * e / r * (2 * q * q - q);
        };
        double lo = 0.3 * sg, hi = lj96_ ? sg : std::pow(2 * s6, 1.0 / 6);   // F(hi) = 0
        if (force(lo) < opt_.force_cap) continue;
        for (int it = 0; it < 80; ++it) {
          const double m = 0.5 * (lo + hi);
          (force(m) > opt_.force_cap ? lo : hi) = m;
        }
        const double r = hi, q = s6 / std::pow(r, 6);
        const double ec = lj96_ ? e * (2 * std::pow(sg / r, 9) - 3 * q) : 4 * e * (q * q - q);
        cap[size_t(a0) * ntab + b0] = make_double4(r * r, ec, force(r), 0.0);
        cap14[size_t(a0) * nt_ + b0] = cap[size_t(a0) * ntab + b0];
      }
  d_tabcap_.upload(cap, stream_);
  d_cap14_.upload(cap14, stream_);
  list_valid_ = false;
  green_valid_ = false;
  if (cell_set_) {
    double c[12];
    std::memcpy(c, cell_h_, sizeof c);
    cell_set_ = false;
    set_cell(c);
  }
  // the active path's PME plans and the mixed path's fixed-point spread grid, also after a switch of precision on an
  // unchanged grid
  ensure_pme();
  CK(cudaStreamSynchronize(stream_));
}

void Engine::set_options(const caps_gpu_opts* o) {
  drop_run_state();
  opt_ = *o;
  setup_options();
}

std::string Engine::capture_state() const {
  std::string k;
  auto put = [&k](const void* p, size_t bytes) { k.append(static_cast<const char*>(p), bytes); };
  const unsigned long long epoch = g_buffer_epoch.load(std::memory_order_relaxed);
  put(&epoch, sizeof epoch);
  put(&opt_, sizeof opt_);
  const int flags[] = {mixed_ ? 1 : 0, energies_ ? 1 : 0, list_valid_ ? 1 : 0, green_valid_ ? 1 : 0, frozen_ ? 1 : 0, batch_tuned_ ? 1 : 0,
                       batch_, pme_lines()[0], pme_lines()[1], pme_lines()[2], nsc_cap_, pk_[0], pk_[1], pk_[2], n_, pair_cut_, pme_cap_, bonded_cap_};
  put(flags, sizeof flags);
  put(cell_h_, sizeof cell_h_);
  put(&dcell_, sizeof dcell_);
  put(&geom_, sizeof geom_);
  return k;
}

// The cell: matrices, list geometry (columns about as wide as a cubic 64-atom super-cluster, reach in columns and
// images as nbnxm.cpp:54-57, 154-161) and the PME grid (kspace.cpp:45-51).
void Engine::set_cell(const double* cell) {
  if (cell_set_ && std::memcmp(cell, cell_h_, sizeof cell_h_) == 0) return;
  std::memcpy(cell_h_, cell, sizeof cell_h_);
  cell_set_ = true;
  cell_matrices(cell, dcell_);
  if (!(dcell_.vol > 0) || !std::isfinite(dcell_.vol)) throw ModelError(CAPS_GPU_EINVAL, "the device path needs a periodic cell with a volume");
  const double* a = cell + 3;
  const double* b = cell + 6;
  const double* c = cell + 9;
  // a frozen pair set keeps its list through a deformation: the images and offsets follow the new cell (the pair
  // kernel and the pack take them from the cell matrix), as the reference's rescale_images (field.cpp:1316-1317)
  const bool keep_list = frozen_;
  double bc[3], ca[3], ab[3];
  cross3(b, c, bc);
  cross3(c, a, ca);
  cross3(a, b, ab);
  ListGeom g{};
  g.w[0] = dcell_.vol / norm3(bc);
  g.w[1] = dcell_.vol / norm3(ca);
  g.w[2] = dcell_.vol / norm3(ab);
  const double side = std::cbrt(64.0 * dcell_.vol / std::max(1, n_));
  g.nu = std::clamp(int(g.w[0] / side), 1, 1024);
  g.nv = std::clamp(int(g.w[1] / side), 1, 1024);
  g.ncol = g.nu * g.nv;
  g.rlist = rc_ + skin_;
  g.rlist2 = g.rlist * g.rlist;
  g.ru = int(std::floor(g.rlist * g.nu / g.w[0])) + 1;
  g.rv = int(std::floor(g.rlist * g.nv / g.w[1])) + 1;
  g.rq = int(std::ceil(g.rlist / g.w[2])) + 1;
  g.dw = g.rlist / g.w[2];
  g.batch = batch_;
  // periodic images in range along each axis: 2 ceil(r_list / w) + 1 for the perpendicular width w (the reference counts
  // the images its bins reach the same way and refuses more than 65536 in all, field.cpp:966-972); the device list also
  // encodes at most +-60 images per axis
  double images = 1;
  for (int d = 0; d < 3; ++d) images *= 2 * std::ceil(g.rlist / g.w[d]) + 1;
  if (images > 65536) throw ModelError(CAPS_GPU_EFIELD, "the cell is too small for the cut-off: more than 65536 periodic images in range");
  if (g.ru / g.nu > 60 || g.rv / g.nv > 60 || g.rq > 60)
    throw ModelError(CAPS_GPU_EFIELD, "the cell is too small for the cut-off: more than 60 periodic images along one axis (the device list's limit)");
  const bool geom_changed = !keep_list && (g.nu != geom_.nu || g.nv != geom_.nv);
  if (!keep_list) geom_ = g;
  if (geom_changed) {
    d_col_count_.alloc(size_t(g.ncol));
    d_col_count_.zero(stream_);   // the scan clears it after every build
    d_col_fill_.alloc(size_t(g.ncol));
    d_col_start_.alloc(size_t(g.ncol) + 1);
    d_col_sc_.alloc(size_t(g.ncol) + 1);
  }
  if (!keep_list) {
    ensure_list_capacity();
    list_valid_ = false;
  }
  green_valid_ = false;
  if (pme_) {
    int k[3];
    const double* e[3] = {a, b, c};
    for (int d = 0; d < 3; ++d) k[d] = good_size(std::max(order_ + 1, int(std::ceil(norm3(e[d]) / opt_.pme_spacing))));
    if (k[0] != pk_[0] || k[1] != pk_[1] || k[2] != pk_[2]) {
      for (int d = 0; d < 3; ++d) pk_[d] = k[d];
      ph1_ = pk_[0] / 2 + 1;
      for (int d = 0; d < 3; ++d) {
        std::vector<double> bsp;
        bspline_moduli(pk_[d], order_, bsp);
        d_bsp_[d].upload(bsp, stream_);
      }
    }
    ensure_pme();
  }
}

void Engine::ensure_list_capacity() {
  const int ncol = geom_.ncol;
  const int nsc = n_ / kScAtoms + ncol + 16;
  // entries: j clusters within the list radius of a super-cluster (its images included), half of them, with margin
  const double dens_cl = double(nsc) * 8.0 / dcell_.vol;
  const double side = std::cbrt(64.0 * dcell_.vol / std::max(1, n_));
  const double R = geom_.rlist + 1.0 * side;
  const double per_sc = 4.0 / 3.0 * kPi * R * R * R * dens_cl;
  const size_t ent = size_t(double(nsc) * std::max(16.0, 0.75 * per_sc)) + 4096;
  if (nsc > nsc_cap_ || ent > d_ent_.n) {
    nsc_cap_ = std::max(nsc, nsc_cap_);
    const size_t ns = size_t(nsc_cap_) * kScAtoms;
    d_sc_col_.alloc(size_t(nsc_cap_));
    d_sc_z_.alloc(size_t(2) * nsc_cap_);
    d_sc_org_.alloc(size_t(3) * nsc_cap_);
    d_cl_box_.alloc(size_t(6) * 8 * nsc_cap_);
    d_cl_real_.alloc(size_t(8) * nsc_cap_);
    d_perm_.alloc(ns);
    d_xq_.alloc(ns);
    d_tslot_.alloc(ns);
    d_Fs_.alloc(3 * ns);
    const size_t ecap = std::max(ent, d_ent_.n);
    d_ent_.alloc(ecap);
    d_ent_shift_.alloc(ecap);
    d_work_.alloc(ecap / 4 + size_t(nsc_cap_) * 2 + 64);
    d_masks_.alloc(size_t(8) * 96 * nsc_cap_ + 8 * 256);   // 8 rows per (j cluster, image) with exclusions, per super-cluster
  }
  if (!mixed_) {   // the FP64 path's packed positions and slot sums, also after a switch of precision
    const size_t ns = size_t(nsc_cap_) * kScAtoms;
    d_xqd_.alloc(ns);
    d_Fsd_.alloc(3 * ns);
  }
  d_col_.alloc(size_t(n_));
  d_frac_.alloc(size_t(3) * n_);
  d_ioff_.alloc(size_t(3) * n_);
  d_order_.alloc(size_t(n_));
  d_iperm_.alloc(size_t(n_));
  d_x0_.alloc(size_t(3) * n_);
  d_xp_.alloc(size_t(3) * n_);
  if (!d_counters_.p) {
    d_counters_.alloc(kCntNum);
    CK(cudaMemsetAsync(d_counters_.p, 0, sizeof(int) * kCntNum, stream_));
    d_errinfo_.alloc(kInfoNum);
    d_errinfo_.zero(stream_);
  }
  d_F_.alloc(size_t(3) * n_);
  if (!mixed_) d_Fd_.alloc(size_t(3) * n_);
  d_efix_.alloc(kENumSlots);
  d_edbl_.alloc(kENumSlots);
  d_x_.alloc(size_t(3) * n_);
  d_f_.alloc(size_t(3) * n_);
  ListBufs& b = lb_;
  b.col = d_col_.p;
  b.frac = d_frac_.p;
  b.ioff = d_ioff_.p;
  b.order = d_order_.p;
  b.iperm = d_iperm_.p;
  b.col_count = d_col_count_.p;
  b.col_fill = d_col_fill_.p;
  b.col_start = d_col_start_.p;
  b.col_sc = d_col_sc_.p;
  b.sc_col = d_sc_col_.p;
  b.sc_z = d_sc_z_.p;
  b.sc_org = d_sc_org_.p;
  b.cl_box = d_cl_box_.p;
  b.cl_real = d_cl_real_.p;
  b.perm = d_perm_.p;
  b.ent = d_ent_.p;
  b.ent_shift = d_ent_shift_.p;
  b.masks = d_masks_.p;
  b.work = d_work_.p;
  b.nsc_cap = nsc_cap_;
  b.ent_cap = int(std::min<size_t>(d_ent_.n, size_t(INT32_MAX)));
  b.mask_cap = int(d_masks_.n / 8);
  b.work_cap = int(d_work_.n);
  b.counters = d_counters_.p;
}

void Engine::check_errors() {
  const unsigned e = unsigned(h_counters_[kCntErr]);
  if (!e) return;
  // the details the failing kernels left (read once, then cleared with the error word and the claims)
  double info[kInfoNum] = {0, 0, 0, 0};
  CK(cudaMemcpy(info, d_errinfo_.p, sizeof info, cudaMemcpyDeviceToHost));
  CK(cudaMemsetAsync(d_counters_.p + kCntErr, 0, sizeof(int), stream_));
  CK(cudaMemsetAsync(d_counters_.p + kCntFeneClaim, 0, 2 * sizeof(int), stream_));
  d_errinfo_.zero(stream_);
  CK(cudaStreamSynchronize(stream_));
  if (e & kErrFene) {   // the reference's text (field.cpp:2157-2159), with the first stretched bond found
    const int b = int(info[kInfoFeneBond]);
    const double r0 = b >= 0 && b < int(h_fene_r0_.size()) ? h_fene_r0_[size_t(b)] : 0.0;
    throw ModelError(CAPS_GPU_EFIELD, "a FENE bond is stretched to r = " + std::to_string(info[kInfoFeneR]) + " Å, past R0 = " + std::to_string(r0) +
                                          " Å; lower --dt or relax the structure first");
  }
  if (e & (kErrListOverflow | kErrMaskOverflow | kErrScOverflow)) throw ModelError(-100, "pair list capacity exceeded");
  if (e & kErrColumnTooBig) throw ModelError(CAPS_GPU_EINVAL, "a grid column holds more atoms than the device sort takes (the cell is too dense or too thin)");
  if (e & kErrExclOverflow) throw ModelError(CAPS_GPU_EINVAL, "too many excluded partners in one super-cluster for the device list");
  if (e & kErrImageRange) throw ModelError(CAPS_GPU_EFIELD, "an excluded pair is more than 63 cells apart: unwrap the molecules first");
  // the reference's texts (constraints.cpp:219, 227, 259)
  if (e & kErrConsOverlap) throw ModelError(CAPS_GPU_ECONSTRAINT, "two constrained atoms sit on each other");
  if (e & (kErrShake | kErrShakeTurn))
    throw ModelError(CAPS_GPU_ECONSTRAINT, (e & kErrShakeTurn) ? "a constrained bond turned by more than 90° in one step; lower the time step or relax first"
                                                                 : "the bond constraints did not converge (SHAKE); lower the time step or relax first");
  if (e & kErrRattle) throw ModelError(CAPS_GPU_ECONSTRAINT, "the bond constraints did not converge (RATTLE); lower the time step");
  // constraints.cpp:131, 182
  if (e & kErrConsOverlap) throw ModelError(CAPS_GPU_ECONSTRAINT, "two constrained atoms sit on each other");
  if (e & kErrLincs) throw ModelError(CAPS_GPU_ECONSTRAINT, "the bond constraints did not converge (LINCS); lower the time step or relax first");
  if (e & kErrFixRange)
    throw ModelError(CAPS_GPU_EFIELD, "a force beyond the fixed-point range (2e9 kcal/mol/Å): overlapping atoms; push the structure off first (FP64 with a force cap)");
  if (e & kErrNonFinite)   // the reference's text (dynamics.cpp:757), with the step whose positions were not finite
    throw ModelError(CAPS_GPU_EFIELD, "the simulation became unstable at step " + std::to_string((long long)info[kInfoNonFiniteStep]) +
                                          "; lower the time step or relax first");
  throw ModelError(CAPS_GPU_EINVAL, "device error word " + std::to_string(e));
}

// Host-side constants: self energy, neutralising background, LJ tail (field.cpp:2455-2537).
void Engine::host_constants(caps_gpu_terms* t, bool ener, bool vir) const {
  (void)vir;
  const bool nonb = (opt_.parts & 2) != 0;
  if (!nonb) return;
  double q2 = 0, qt = 0;
  for (double c : h_q_) q2 += c * c, qt += c;
  if (coul_) {
    if (pme_) {
      if (ener) t->coulomb -= kCoulomb * beta_ / std::sqrt(kPi) * q2;
      if (std::fabs(qt) > 1e-10) {
        const double eb = -kCoulomb * kPi * qt * qt / (2 * dcell_.vol * beta_ * beta_);
        if (ener) t->coulomb += eb;
        t->virial += 3 * eb;
        for (int c = 0; c < 3; ++c) t->w[c] += eb;
      }
    } else if (ener) {
      const double a = opt_.dsf_alpha;
      t->coulomb -= (erfc_rc_ / (2 * rc_) + dsf_f0_ * rc_ / 2 + a / std::sqrt(kPi)) * q2 * kCoulomb;
    }
  }
  if (tail_) {
    const double vol = dcell_.vol, rc2 = rc_ * rc_, rc3 = rc2 * rc_, rc9 = rc3 * rc3 * rc3;
    double et = 0, wt = 0;
    for (int a0 = 0; a0 < nt_; ++a0)
      for (int b0 = 0; b0 < nt_; ++b0) {
        const double eps = h_eps_[size_t(a0) * nt_ + b0], s6 = std::pow(h_sig_[size_t(a0) * nt_ + b0], 6), s12 = s6 * s6;
        const double nn = type_count_[size_t(a0)] * type_count_[size_t(b0)];
        const size_t tp = size_t(a0) * nt_ + b0;
        if (h_form_[tp] == 1) {   // Buckingham, as LAMMPS pair buck (field.cpp:2508-2514)
          const double A = h_pa_[tp], rho = h_pb_[tp], Cc = h_pc_[tp], ex = std::exp(-rc_ / rho);
          et += nn * 2 * kPi * (A * rho * ex * (rc2 + 2 * rho * rc_ + 2 * rho * rho) - Cc / (3 * rc3));
          wt += nn * 2 * kPi * (A * ex * (rc3 + 3 * rho * rc2 + 6 * rho * rho * rc_ + 6 * rho * rho * rho) - 2 * Cc / rc3);
          continue;
        }
        if (h_form_[tp] == 2 || h_form_[tp] == 3) continue;   // Morse, Rydberg: no tail term
        if (h_form_[tp] == 13) {   // a 12-6 SDK pair: its own 12-6 tail (field.cpp:2516-2521)
          const double e6 = h_pa_[tp], sg6 = std::pow(h_pb_[tp], 6), sg12 = sg6 * sg6;
          et += nn * 2 * kPi * 4 * e6 * (sg12 / (9 * rc9) - sg6 / (3 * rc3));
          wt += nn * 2 * kPi * 4 * e6 * (4 * sg12 / (3 * rc9) - 2 * sg6 / rc3);
          continue;
        }
        if (h_form_[tp] >= 11) continue;   // the other SDK forms, lj/gromacs, cosine-squared, tables: none
        if (lj96_) {   // lj/class2 (field.cpp:2523-2529)
          const double s3 = std::sqrt(s6), rc6 = rc3 * rc3;
          et += nn * 2 * kPi * eps * s6 * (s3 - 3 * rc3) / (3 * rc6);
          wt += nn * 3 * 2 * kPi * eps * s6 * (s3 - 2 * rc3) / rc6;
          continue;
        }
        et += nn * 2 * kPi * 4 * eps * (s12 / (9 * rc9) - s6 / (3 * rc3));
        wt += nn * 2 * kPi * 4 * eps * (4 * s12 / (3 * rc9) - 2 * s6 / rc3);
      }
    if (ener) t->vdw += et / vol;
    t->virial += wt / vol;
    t->tail_energy = et / vol;
    t->tail_virial = wt / vol;
    for (int c = 0; c < 3; ++c) t->w[c] += wt / vol / 3;
  }
}

void Engine::read_terms(caps_gpu_terms* out, bool ener, bool vir) {
  caps_gpu_terms t{};
  double e[kENumSlots];
  for (int k = 0; k < kENumSlots; ++k) e[k] = mixed_ ? double(h_efix_[k]) * kInvFixE : h_edbl_[k];
  t.bond = e[kEBond];
  t.angle = e[kEAngle];
  t.dihedral = e[kEDihedral];
  t.improper = e[kEImproper];
  t.vdw = e[kEVdw];
  t.coulomb = e[kECoul];
  for (int c = 0; c < 6; ++c) t.w[c] = vir ? e[kEW0 + c] : 0.0;
  t.virial = t.w[0] + t.w[1] + t.w[2];
  host_constants(&t, ener, vir);
  if (out) *out = t;
}

// The pair list's entry, shift, work-item and exclusion-mask buffers made large enough for `ent` entries and `mk` mask
// words; the next evaluation builds the list again.
void Engine::grow_list(size_t ent, size_t mk) {
  if (ent > d_ent_.n) {
    d_ent_.release();
    d_ent_shift_.release();
    d_ent_.alloc(ent);
    d_ent_shift_.alloc(ent);
    d_work_.release();
    d_work_.alloc(ent / 4 + size_t(nsc_cap_) * 2 + 64);
  }
  if (mk > d_masks_.n) {
    d_masks_.release();
    d_masks_.alloc(mk);
  }
  ensure_list_capacity();
  list_valid_ = false;
}

// After the first evaluation of a run (synchronises): a list that overflowed its buffers, or filled more than two
// thirds of them, is given room for 1.5 times what it holds (twice its capacity after an overflow), since a run's
// list grows with the density it reaches and an overflow within a run ends the run. True: the list must be built again.
bool Engine::grow_list_for_run() {
  CK(cudaMemcpyAsync(h_counters_, d_counters_.p, sizeof(int) * kCntNum, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  const unsigned e = unsigned(h_counters_[kCntErr]);
  const bool over = (e & (kErrListOverflow | kErrMaskOverflow)) != 0;
  const size_t used_e = size_t(std::max(0, h_counters_[kCntEnt])), used_m = size_t(std::max(0, h_counters_[kCntMask])) * 8;
  size_t ent = d_ent_.n, mk = d_masks_.n;
  if (over || 3 * used_e > 2 * d_ent_.n) ent = std::max(over ? 2 * d_ent_.n : d_ent_.n, used_e + used_e / 2);
  if (over || 3 * used_m > 2 * d_masks_.n) mk = std::max(over ? 2 * d_masks_.n : d_masks_.n, used_m + used_m / 2);
  if (ent == d_ent_.n && mk == d_masks_.n) return false;
  if (over) {   // the overflow is answered here: clear it for the evaluation that follows
    CK(cudaMemsetAsync(d_counters_.p + kCntErr, 0, sizeof(int), stream_));
    h_counters_[kCntErr] = 0;
  }
  grow_list(ent, mk);
  return true;
}

void Engine::compute_dev(const double* d_x, const double* cell, double* d_f, caps_gpu_terms* out) {
  set_cell(cell);
  for (int attempt = 0;; ++attempt) {
    forces(d_x, true, true, true);
    CK(cudaMemcpyAsync(h_counters_, d_counters_.p, sizeof(int) * kCntNum, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(h_efix_, d_efix_.p, sizeof(long long) * kENumSlots, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(h_edbl_, d_edbl_.p, sizeof(double) * kENumSlots, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    try {
      check_errors();
    } catch (const ModelError& m) {
      if (m.code != -100 || attempt >= 3) throw;
      grow_list(d_ent_.n * 2, d_masks_.n * 2);   // and build again
      continue;
    }
    break;
  }
  const bool ener_pairs = energies_ || !mixed_;
  (void)ener_pairs;
  read_terms(out, true, true);
  if (d_f != d_f_.p) CK(cudaMemcpyAsync(d_f, d_f_.p, sizeof(double) * 3 * size_t(n_), cudaMemcpyDeviceToDevice, stream_));
  CK(cudaStreamSynchronize(stream_));
}

void Engine::compute_host(const double* x, const double* cell, double* f, caps_gpu_terms* out) {
  for (size_t k = 0; k < size_t(3) * n_; ++k)
    if (!std::isfinite(x[k])) throw ModelError(CAPS_GPU_EFIELD, "non-finite coordinates: atom " + std::to_string(k / 3 + 1));
  set_cell(cell);
  CK(cudaMemcpyAsync(d_x_.p, x, sizeof(double) * 3 * size_t(n_), cudaMemcpyHostToDevice, stream_));
  compute_dev(d_x_.p, cell, d_f_.p, out);
  CK(cudaMemcpyAsync(f, d_f_.p, sizeof(double) * 3 * size_t(n_), cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
}


}  // namespace capsb

// ---------------------------------------------------------------------------------------------------------------
// C ABI
using capsb::Engine;

struct caps_gpu_engine {
  std::unique_ptr<Engine> e;
  std::string err;
};

namespace {
thread_local std::string g_create_error;
}  // namespace

namespace capsb {
// The text caps_gpu_error(NULL) returns, for calls that fail without an engine.
void set_call_error(const std::string& text) { g_create_error = text; }
}  // namespace capsb

namespace {

int32_t guard(caps_gpu_engine* h, const std::function<void()>& fn) {
  try {
    fn();
    return CAPS_GPU_OK;
  } catch (const capsb::ModelError& m) {
    if (h) h->err = m.what();
    else g_create_error = m.what();
    return m.code < 0 && m.code > -100 ? m.code : CAPS_GPU_EINVAL;
  } catch (const capsb::CudaError& c) {
    if (h) h->err = c.what();
    else g_create_error = c.what();
    return CAPS_GPU_ECUDA;
  } catch (const std::exception& x) {
    if (h) h->err = x.what();
    else g_create_error = x.what();
    return CAPS_GPU_EINVAL;
  }
}
}  // namespace

extern "C" {

int32_t caps_gpu_abi_version(void) { return CAPS_GPU_ABI_VERSION; }

int32_t caps_gpu_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

caps_gpu_engine* caps_gpu_create(const caps_gpu_ff* ff, const caps_gpu_opts* opts) {
  if (!ff || !opts) {
    g_create_error = "caps_gpu_create: null argument";
    return nullptr;
  }
  auto h = std::make_unique<caps_gpu_engine>();
  const int32_t rc = guard(nullptr, [&] { h->e = std::make_unique<Engine>(ff, opts); });
  if (rc != CAPS_GPU_OK) return nullptr;
  return h.release();
}

int32_t caps_gpu_set_options(caps_gpu_engine* e, const caps_gpu_opts* opts) {
  if (!e || !opts) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->set_options(opts); });
}

int32_t caps_gpu_energies(caps_gpu_engine* e, int32_t on) {
  if (!e) return CAPS_GPU_EINVAL;
  e->e->energies(on != 0);
  return CAPS_GPU_OK;
}

int32_t caps_gpu_compute(caps_gpu_engine* e, const double* x, const double* cell, double* f, caps_gpu_terms* out) {
  if (!e || !x || !cell || !f) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->compute_host(x, cell, f, out); });
}

int32_t caps_gpu_compute_device(caps_gpu_engine* e, const double* d_x, const double* cell, double* d_f, caps_gpu_terms* out) {
  if (!e || !d_x || !cell || !d_f) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->compute_dev(d_x, cell, d_f, out); });
}

int32_t caps_gpu_reload(caps_gpu_engine* e, const caps_gpu_ff* ff) {
  if (!e || !ff) return CAPS_GPU_EINVAL;
  return guard(e, [&] {
    Engine& old = *e->e;
    if (ff->natoms != old.n_) throw capsb::ModelError(CAPS_GPU_EINVAL, "reload: the force field has another number of atoms");
    caps_gpu_opts o = old.opt_;
    if (old.frozen()) old.unfreeze();   // reload ends a frozen list (field.cpp:432), and restores the precision it switched
    o = old.opt_;
    auto fresh = std::make_unique<Engine>(ff, &o);
    fresh->energies(old.energies_on());
    fresh->set_timing(old.timing_flush());
    e->e = std::move(fresh);
  });
}

int32_t caps_gpu_freeze_pairs(caps_gpu_engine* e, const double* x, const double* cell) {
  if (!e || !x || !cell) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->freeze_pairs(x, cell); });
}

int32_t caps_gpu_unfreeze(caps_gpu_engine* e) {
  if (!e) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->unfreeze(); });
}

int64_t caps_gpu_pairs(caps_gpu_engine* e) {
  if (!e) return -1;
  try {
    return e->e->pairs();
  } catch (const std::exception& x) {
    e->err = x.what();
    return -1;
  }
}

int32_t caps_gpu_threads(const caps_gpu_engine* e) { return e ? e->e->sms() : 0; }

int32_t caps_gpu_list_builds(const caps_gpu_engine* e) {
  if (!e) return 0;
  try {
    return e->e->list_builds();
  } catch (...) {
    return -1;
  }
}

int32_t caps_gpu_run(caps_gpu_engine* e, caps_gpu_state* state, const caps_gpu_md_opts* md, caps_gpu_progress_fn progress, caps_gpu_frame_fn frame,
                     void* user, char* report, int32_t report_cap) {
  if (!e || !state || !md || !state->x || !state->cell) return CAPS_GPU_EINVAL;
  std::string rep;
  const int32_t rc = guard(e, [&] { e->e->run(state, md, progress, frame, user, &rep); });
  if (report && report_cap > 0) {
    std::snprintf(report, size_t(report_cap), "%s", rc == CAPS_GPU_OK ? rep.c_str() : e->err.c_str());
  }
  return rc;
}

int32_t caps_gpu_run_batch(caps_gpu_engine* const* engines, caps_gpu_state* const* states, const caps_gpu_md_opts* const* md, int32_t count,
                           caps_gpu_progress_fn progress, caps_gpu_frame_fn frame, void* const* user) {
  if (!engines || !states || !md || count < 1) return CAPS_GPU_EINVAL;
  std::vector<capsb::Engine*> es;
  for (int32_t r = 0; r < count; ++r) {
    if (!engines[r] || !states[r] || !md[r] || !states[r]->x || !states[r]->cell) return CAPS_GPU_EINVAL;
    for (int32_t q = 0; q < r; ++q)
      if (engines[q] == engines[r]) {
        engines[0]->err = "caps_gpu_run_batch: an engine appears twice in the batch";
        return CAPS_GPU_EINVAL;
      }
    es.push_back(engines[r]->e.get());
  }
  return guard(engines[0], [&] { capsb::run_batch(es, states, md, progress, frame, user); });
}

double caps_gpu_last_steps_per_second(const caps_gpu_engine* e) { return e ? e->e->last_steps_per_second() : 0.0; }

void caps_gpu_destroy(caps_gpu_engine* e) { delete e; }

int32_t caps_gpu_diag_set_timing(caps_gpu_engine* e, int64_t flush_bytes) {
  if (!e) return CAPS_GPU_EINVAL;
  e->e->set_timing(flush_bytes);
  return CAPS_GPU_OK;
}

int32_t caps_gpu_diag_get_tuning(const caps_gpu_engine* e, int32_t* v) {
  if (!e || !v) return CAPS_GPU_EINVAL;
  e->e->tuning(v);
  return CAPS_GPU_OK;
}

int32_t caps_gpu_diag_set_tuning(caps_gpu_engine* e, const int32_t* v) {
  if (!e || !v) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->pin_tuning(v); });
}

double caps_gpu_diag_last_step_ms(const caps_gpu_engine* e) { return e ? e->e->last_step_ms_device() : 0.0; }

int32_t caps_gpu_diag_step_kernels(const caps_gpu_engine* e) { return e ? e->e->graph_kernels() : 0; }
int64_t caps_gpu_diag_kernels_run(const caps_gpu_engine* e) { return e ? e->e->kernels_run() : 0; }
int32_t caps_gpu_diag_list_counts(caps_gpu_engine* e, int64_t* v) {
  if (!e || !v) return CAPS_GPU_EINVAL;
  return guard(e, [&] {
    e->e->list_counts(v);
  });
}

int32_t caps_gpu_diag_pair_timing(caps_gpu_engine* e, const double* x, const double* cell, int32_t launches, int64_t flush_bytes, double* avg_ms,
                                  double* pairs_in, double* pairs_listed, double* entries) {
  if (!e || !x || !cell || launches < 1) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->time_pair_kernel(x, cell, launches, flush_bytes, avg_ms, pairs_in, pairs_listed, entries); });
}

int32_t caps_gpu_diag_phase_timing(caps_gpu_engine* e, const double* x, const double* cell, int32_t launches, int64_t flush_bytes, double* ms) {
  if (!e || !x || !cell || !ms || launches < 1) return CAPS_GPU_EINVAL;
  return guard(e, [&] { e->e->time_phases(x, cell, launches, flush_bytes, ms); });
}

const char* caps_gpu_error(const caps_gpu_engine* e) { return e ? e->err.c_str() : g_create_error.c_str(); }

}  // extern "C"
