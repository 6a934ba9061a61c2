// ORACLE / TEST INFRASTRUCTURE — not part of the product path.
//
// A C entry layer over the reference CAPS C++ core (compiled from its sources by oracle/Makefile), so that the parity
// tests and the CPU baseline can drive the reference from plain arrays through ctypes. It takes the same POD force
// field (caps_gpu_ff, include/caps_gpu.h) the device engine takes and rebuilds a caps::ForceField from it:
//   ref_compute  -> caps::Evaluator::compute      (core/src/field.cpp:1249)
//   ref_run      -> caps::run_dynamics            (core/src/dynamics.cpp:71)
//   ref_pme      -> caps::pme_reciprocal (threaded, core/src/kspace.cpp:80)
//   ref_fit_tg   -> caps::fit_bilinear / caps::fit_two_ranges (core/src/mechanics.cpp:1218, 1310)
//   ref_run_cooling -> caps::run_cooling      (core/src/mechanics.cpp:1381)
//   ref_equilibrate -> caps::equilibrate      (core/src/equilibrate.cpp:199)
//   ref_minimise -> caps::minimise              (core/src/relax.cpp:65)
//   ref_build_*  -> the reference builders (grow + relax + assign_gaff as tests/test_nbnxm.cpp:19-34; kremer_grest),
//                   written to a flat binary file the Python side reads (tests/golden fixtures are made from these).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "caps/dynamics.hpp"
#include "caps/field.hpp"
#include "caps/grow.hpp"
#include "caps/io.hpp"
#include "caps/live.hpp"
#include "caps/kremer_grest.hpp"
#include "caps/kspace.hpp"
#include "caps/mechanics.hpp"
#include "caps/equilibrate.hpp"
#include "caps/relax.hpp"
#include "kspace_pool.hpp"
#include "parallel.hpp"
#include "caps_gpu.h"

using namespace caps;

namespace {

thread_local std::string g_err;

Cell to_cell(const double* c) {
  Cell cell;
  for (int k = 0; k < 3; ++k) {
    cell.origin[k] = c[k];
    cell.a[k] = c[3 + k];
    cell.b[k] = c[6 + k];
    cell.c[k] = c[9 + k];
  }
  return cell;
}

void from_cell(const Cell& cell, double* c) {
  for (int k = 0; k < 3; ++k) {
    c[k] = cell.origin[k];
    c[3 + k] = cell.a[k];
    c[6 + k] = cell.b[k];
    c[9 + k] = cell.c[k];
  }
}

std::shared_ptr<ForceField> to_ff(const caps_gpu_ff* p) {
  auto ff = std::make_shared<ForceField>();
  const int n = p->natoms, nt = p->ntypes;
  ff->name = "from caps_gpu_ff";
  ff->type_index.assign(p->type_index, p->type_index + n);
  ff->atom_type.resize(size_t(n));
  ff->type_names.resize(size_t(nt));
  ff->lj.assign(size_t(nt), PairType{0.0, 1.0});
  for (int t = 0; t < nt; ++t) {
    ff->type_names[size_t(t)] = "t" + std::to_string(t);
    ff->lj[size_t(t)] = {p->pair_eps[t * nt + t], p->pair_sigma[t * nt + t]};
  }
  for (int i = 0; i < n; ++i) ff->atom_type[size_t(i)] = ff->type_names[size_t(p->type_index[i])];
  for (int a = 0; a < nt; ++a)
    for (int b = a; b < nt; ++b) ff->pair_override[{a, b}] = PairType{p->pair_eps[a * nt + b], p->pair_sigma[a * nt + b]};
  ff->mixing = "geometric";
  ff->pair_form = p->lj_form == 1 ? "lj9-6" : "lj12-6";
  for (int k = 0; k < p->npair_func; ++k) {
    const double* q = p->pair_func_p + 5 * k;
    PairFunc f;
    f.form = int(q[0]);
    f.a = q[1], f.b = q[2], f.c = q[3], f.rc = q[4];
    ff->pair_func[{p->pair_func_ab[2 * k], p->pair_func_ab[2 * k + 1]}] = f;
  }
  ff->lj_inner = p->lj_inner;
  ff->lj_fsw = p->lj_fsw != 0;
  for (int k = 0, off = 0; k < p->ntables; ++k) {
    TabulatedPair tb;
    tb.r0 = p->table_r0_dr[2 * k];
    tb.dr = p->table_r0_dr[2 * k + 1];
    tb.e.assign(p->table_e + off, p->table_e + off + p->table_n[k]);
    tb.f.assign(p->table_f + off, p->table_f + off + p->table_n[k]);
    off += p->table_n[k];
    ff->tables.push_back(std::move(tb));
  }
  ff->charge.assign(p->charge, p->charge + n);
  ff->mass.assign(p->mass, p->mass + n);
  for (int k = 0; k < p->nbonds; ++k) ff->bonds.push_back({p->bond_ij[2 * k], p->bond_ij[2 * k + 1], p->bond_k_r0[2 * k], p->bond_k_r0[2 * k + 1]});
  for (int k = 0; k < p->nangles; ++k)
    ff->angles.push_back({p->angle_ijk[3 * k], p->angle_ijk[3 * k + 1], p->angle_ijk[3 * k + 2], p->angle_kt_theta0[2 * k], p->angle_kt_theta0[2 * k + 1]});
  for (int k = 0; k < p->ndihedrals; ++k)
    ff->dihedrals.push_back({p->dihedral_ijkl[4 * k], p->dihedral_ijkl[4 * k + 1], p->dihedral_ijkl[4 * k + 2], p->dihedral_ijkl[4 * k + 3],
                             p->dihedral_v_delta[2 * k], p->dihedral_n[k], p->dihedral_v_delta[2 * k + 1]});
  for (int k = 0; k < p->nimpropers; ++k)
    ff->impropers.push_back({p->improper_ijkl[4 * k], p->improper_ijkl[4 * k + 1], p->improper_ijkl[4 * k + 2], p->improper_ijkl[4 * k + 3],
                             p->improper_v_delta[2 * k], p->improper_n[k], p->improper_v_delta[2 * k + 1]});
  for (int k = 0; k < p->npairs14; ++k) {
    ff->pairs14.push_back({p->pair14_ij[2 * k], p->pair14_ij[2 * k + 1]});
    if (p->pair14_lj) ff->pairs14_lj.push_back(p->pair14_lj[k]);
    if (p->pair14_coul) ff->pairs14_coul.push_back(p->pair14_coul[k]);
  }
  if (p->pair14_lj && !p->pair14_coul) ff->pairs14_coul.assign(size_t(p->npairs14), p->coul14);
  if (p->pair14_coul && !p->pair14_lj) ff->pairs14_lj.assign(size_t(p->npairs14), p->lj14);
  ff->lj14 = p->lj14;
  ff->coul14 = p->coul14;
  ff->excluded.assign(size_t(n), {});
  if (p->excl_offset)
    for (int i = 0; i < n; ++i) ff->excluded[size_t(i)].assign(p->excl_list + p->excl_offset[i], p->excl_list + p->excl_offset[i + 1]);
  for (int k = 0; k < p->nfene; ++k) {
    const double* q = p->fene_k_r0_eps_sigma + 4 * k;
    ff->bonds_x.push_back({p->fene_ij[2 * k], p->fene_ij[2 * k + 1], 3, q[0], q[1], q[2], q[3]});
  }
  ff->lj_shift = p->lj_shift != 0;
  ff->cutoff = p->model_cutoff;
  return ff;
}

EnergyOptions to_eo(const caps_gpu_opts* o, int threads) {
  EnergyOptions e;
  e.cutoff = o->cutoff;
  e.skin = o->skin;
  e.coulomb = o->coulomb != 0;
  e.electrostatics = o->electrostatics ? EnergyOptions::Electrostatics::PME : EnergyOptions::Electrostatics::DSF;
  e.dsf_alpha = o->dsf_alpha;
  e.ewald_rtol = o->ewald_rtol;
  e.pme_spacing = o->pme_spacing;
  e.pme_order = o->pme_order;
  e.tail = o->tail != 0;
  e.mixed = o->precision == 0;
  e.force_cap = o->force_cap;
  e.parts = o->parts ? o->parts : 3;
  e.threads = threads;
  return e;
}

void to_terms(const EnergyTerms& t, caps_gpu_terms* o) {
  o->bond = t.bond;
  o->angle = t.angle;
  o->dihedral = t.dihedral;
  o->improper = t.improper;
  o->vdw = t.vdw;
  o->coulomb = t.coulomb;
  o->virial = t.virial;
  for (int c = 0; c < 6; ++c) o->w[c] = t.w[c];
  o->tail_energy = t.tail_energy;
  o->tail_virial = t.tail_virial;
}

// --- a flat binary export: records of (name[32], kind char, 7 pad bytes, int64 count, data) ---------------------
struct Writer {
  FILE* f;
  explicit Writer(const char* path) : f(std::fopen(path, "wb")) {
    if (!f) throw std::runtime_error(std::string("cannot write ") + path);
    std::fwrite("CAPSFF1\n", 1, 8, f);
  }
  ~Writer() { if (f) std::fclose(f); }
  void rec(const char* name, char kind, const void* data, int64_t count, size_t size) {
    char head[40] = {0};
    std::strncpy(head, name, 31);
    head[32] = kind;
    std::fwrite(head, 1, 40, f);
    std::fwrite(&count, sizeof count, 1, f);
    if (count) std::fwrite(data, size, size_t(count), f);
  }
  void d(const char* name, const std::vector<double>& v) { rec(name, 'd', v.data(), int64_t(v.size()), 8); }
  void i(const char* name, const std::vector<int32_t>& v) { rec(name, 'i', v.data(), int64_t(v.size()), 4); }
  void u(const char* name, const std::vector<uint32_t>& v) { rec(name, 'u', v.data(), int64_t(v.size()), 4); }
  void s(const char* name, const std::string& v) { rec(name, 's', v.data(), int64_t(v.size()), 1); }
};

void export_system(const System& s, const ForceField& ff, const char* path) {
  Writer w(path);
  const size_t n = s.atoms.size(), nt = ff.lj.size();
  std::vector<double> x, cell(12);
  for (const auto& a : s.atoms) x.insert(x.end(), a.pos.begin(), a.pos.end());
  from_cell(s.cell, cell.data());
  w.d("x", x);
  w.d("cell", cell);
  std::vector<int32_t> el, ti(ff.type_index.begin(), ff.type_index.end());
  for (const auto& a : s.atoms) el.push_back(a.element);
  w.i("element", el);
  w.i("type_index", ti);
  w.d("charge", ff.charge);
  w.d("mass", ff.mass);
  std::vector<double> pe(nt * nt), ps(nt * nt);
  for (size_t a = 0; a < nt; ++a)
    for (size_t b = 0; b < nt; ++b) {
      const PairType pt = mixed_pair(ff, int(a), int(b));
      pe[a * nt + b] = pt.eps;
      ps[a * nt + b] = pt.sigma;
    }
  w.d("pair_eps", pe);
  w.d("pair_sigma", ps);
  std::vector<uint32_t> bij;
  std::vector<double> bkr;
  for (const auto& b : ff.bonds) bij.insert(bij.end(), {b.i, b.j}), bkr.insert(bkr.end(), {b.k, b.r0});
  w.u("bond_ij", bij);
  w.d("bond_k_r0", bkr);
  std::vector<uint32_t> aijk;
  std::vector<double> akt;
  for (const auto& a : ff.angles) aijk.insert(aijk.end(), {a.i, a.j, a.k}), akt.insert(akt.end(), {a.kt, a.theta0});
  w.u("angle_ijk", aijk);
  w.d("angle_kt_theta0", akt);
  auto tors = [&](const std::vector<TorsionTerm>& T, const char* a, const char* b, const char* c) {
    std::vector<uint32_t> ijkl;
    std::vector<double> vd;
    std::vector<int32_t> nn;
    for (const auto& t : T) ijkl.insert(ijkl.end(), {t.i, t.j, t.k, t.l}), vd.insert(vd.end(), {t.v, t.delta}), nn.push_back(t.n);
    w.u(a, ijkl);
    w.d(b, vd);
    w.i(c, nn);
  };
  tors(ff.dihedrals, "dihedral_ijkl", "dihedral_v_delta", "dihedral_n");
  tors(ff.impropers, "improper_ijkl", "improper_v_delta", "improper_n");
  std::vector<uint32_t> p14;
  for (const auto& p : ff.pairs14) p14.insert(p14.end(), {p[0], p[1]});
  w.u("pair14_ij", p14);
  w.d("pair14_lj", ff.pairs14_lj);
  w.d("pair14_coul", ff.pairs14_coul);
  w.d("lj14_coul14", {ff.lj14, ff.coul14});
  std::vector<uint32_t> eo{0}, el2;
  for (size_t i = 0; i < n; ++i) {
    const auto& e = i < ff.excluded.size() ? ff.excluded[i] : std::vector<uint32_t>{};
    el2.insert(el2.end(), e.begin(), e.end());
    eo.push_back(uint32_t(el2.size()));
  }
  w.u("excl_offset", eo);
  w.u("excl_list", el2);
  std::vector<uint32_t> fij;
  std::vector<double> fp;
  int other_bx = 0;
  for (const auto& b : ff.bonds_x) {
    if (b.form != 3) { ++other_bx; continue; }
    fij.insert(fij.end(), {b.i, b.j});
    fp.insert(fp.end(), {b.a, b.b, b.c, b.d});
  }
  w.u("fene_ij", fij);
  w.d("fene_k_r0_eps_sigma", fp);
  w.i("flags", {ff.lj_shift ? 1 : 0, ff.keep13 ? 1 : 0});
  w.d("model_cutoff", {ff.cutoff});
  // terms the device path does not take: the exporter counts them so a test can refuse such a cell
  const size_t unsupported = ff.impropers_harmonic.size() + ff.inversions.size() + size_t(other_bx) + ff.angles_x.size() + ff.urey_bradley.size() +
                             ff.cbt.size() + ff.lj_pairs.size() + ff.pair_func.size() + ff.bonds2.size() + ff.angles2.size() + ff.dihedrals2.size() +
                             ff.impropers2.size() + ff.vsites.size() + (ff.pair_form != "lj12-6") + ff.lj14_types.size();
  w.i("unsupported", {int32_t(unsupported)});
  w.s("name", ff.name);
}

System to_system(const caps_gpu_ff* p, const std::shared_ptr<ForceField>& ff, const caps_gpu_state* st, const int32_t* element) {
  System s;
  const int n = p->natoms;
  s.atoms.resize(size_t(n));
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) s.atoms[size_t(i)].pos[k] = st->x[3 * i + k];
    s.atoms[size_t(i)].element = element ? element[i] : 6;
    s.atoms[size_t(i)].charge = p->charge[i];
    s.atoms[size_t(i)].type = p->type_index[i] + 1;
  }
  for (const auto& b : ff->bonds) s.bonds.push_back({b.i, b.j, 1});
  for (const auto& b : ff->bonds_x) s.bonds.push_back({b.i, b.j, 1});
  // the types' masses, as a data file's Masses section gives them (System::mass_of reads these before element masses)
  std::vector<char> seen(size_t(p->ntypes), 0);
  for (int i = 0; i < n; ++i) {
    const int t = p->type_index[i];
    if (t < 0 || t >= p->ntypes || seen[size_t(t)]) continue;
    seen[size_t(t)] = 1;
    TypeInfo ti;
    ti.type = t + 1;
    ti.mass = p->mass[i];
    s.types.push_back(ti);
  }
  s.cell = to_cell(st->cell);
  if (st->has_velocities && st->v) {
    s.velocities.resize(size_t(n));
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) s.velocities[size_t(i)][k] = st->v[3 * i + k];
  }
  return s;
}

// The reference's BilinearFit (core/include/caps/mechanics.hpp:303-311) as a POD for ctypes.
typedef struct {
  int32_t ok;
  double tg, tg_err, slope_low, slope_high, value_at_tg, alpha_low, alpha_high, rss;
  char note[256];
} ref_tg_fit;

void to_fit(const BilinearFit& f, ref_tg_fit* out) {
  std::memset(out, 0, sizeof *out);
  out->ok = f.ok ? 1 : 0;
  out->tg = f.tg, out->tg_err = f.tg_err, out->slope_low = f.slope_low, out->slope_high = f.slope_high;
  out->value_at_tg = f.value_at_tg, out->alpha_low = f.alpha_low, out->alpha_high = f.alpha_high, out->rss = f.rss;
  std::strncpy(out->note, f.note.c_str(), sizeof out->note - 1);
}

}  // namespace

extern "C" {

const char* ref_error() { return g_err.c_str(); }

int ref_compute(const caps_gpu_ff* p, const caps_gpu_opts* o, const double* x, const double* cell, double* f, caps_gpu_terms* out, int threads) {
  try {
    auto ff = to_ff(p);
    Evaluator ev(*ff, to_eo(o, threads));
    std::vector<double> xv(x, x + 3 * size_t(p->natoms)), fv;
    const EnergyTerms t = ev.compute(xv, to_cell(cell), fv);
    std::memcpy(f, fv.data(), fv.size() * sizeof(double));
    to_terms(t, out);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// Times `reps` evaluations on one evaluator (the list built on the first), for the CPU baseline: seconds per call.
int ref_time_compute(const caps_gpu_ff* p, const caps_gpu_opts* o, const double* x, const double* cell, int reps, int threads, double* seconds) {
  try {
    auto ff = to_ff(p);
    Evaluator ev(*ff, to_eo(o, threads));
    std::vector<double> xv(x, x + 3 * size_t(p->natoms)), fv;
    const Cell c = to_cell(cell);
    ev.compute(xv, c, fv);
    const auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < reps; ++r) ev.compute(xv, c, fv);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / std::max(1, reps);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// run_dynamics on a System rebuilt from the arrays. element: [natoms] atomic numbers (for SHAKE's hydrogens and rigid
// waters). rows: up to max_rows thermo rows out. seconds and ns_per_day from the reference's own report.
// frame (may be NULL): each recorded frame with `user`; md->checkpoint (may be NULL): each checkpoint. A stop asked for
// with ref_request_stop ends the run with DynamicsInterrupted: the state is written back and 1 returned.
int ref_run(const caps_gpu_ff* p, const caps_gpu_opts* eo, caps_gpu_state* st, const caps_gpu_md_opts* md, const int32_t* element, int threads,
            caps_gpu_thermo* rows, int max_rows, int* nrows, double* seconds, double* ns_per_day, caps_gpu_frame_fn frame, void* user) {
  try {
    auto ff = to_ff(p);
    System s;
    const int n = p->natoms;
    s.atoms.resize(size_t(n));
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) s.atoms[size_t(i)].pos[k] = st->x[3 * i + k];
      s.atoms[size_t(i)].element = element ? element[i] : 6;
      s.atoms[size_t(i)].charge = p->charge[i];
      s.atoms[size_t(i)].type = p->type_index[i] + 1;
    }
    for (const auto& b : ff->bonds) s.bonds.push_back({b.i, b.j, 1});
    for (const auto& b : ff->bonds_x) s.bonds.push_back({b.i, b.j, 1});
    s.cell = to_cell(st->cell);
    if (st->has_velocities && st->v) {
      s.velocities.resize(size_t(n));
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) s.velocities[size_t(i)][k] = st->v[3 * i + k];
    }
    DynamicsOptions o;
    o.field = ff;
    o.dt = md->dt;
    o.steps = md->steps;
    o.temperature = md->temperature;
    o.temperature_end = md->temperature_end;
    const Thermostat th[4] = {Thermostat::None, Thermostat::Bussi, Thermostat::Langevin, Thermostat::NoseHoover};
    o.thermostat = th[md->thermostat & 3];
    o.tau_t = md->tau_t;
    o.barostat = md->barostat == 1 ? Barostat::CRescale : md->barostat == 2 ? Barostat::Berendsen : md->barostat == 3 ? Barostat::MTK : Barostat::None;
    o.pressure = md->pressure;
    o.tau_p = md->tau_p;
    o.compressibility = md->compressibility;
    o.barostat_every = md->barostat_every;
    o.hmr = md->hmr;
    o.anisotropic = md->anisotropic != 0;
    for (int a = 0; a < 3; ++a) {
      o.couple_axis[a] = md->couple_axes == 0 || ((md->couple_axes >> a) & 1);
      if ((md->axis_pressure_set >> a) & 1) o.axis_pressure[a] = md->axis_pressure[a];
    }
    o.constraints = md->constraints ? ConstraintMode::HBonds : ConstraintMode::None;
    o.constraint_algorithm = md->constraint_algorithm == 1 ? ConstraintAlgorithm::Lincs : ConstraintAlgorithm::Shake;
    o.new_velocities = md->new_velocities != 0;
    o.seed = md->seed;
    o.thermo_every = md->thermo_every;
    o.frame_every = frame ? md->frame_every : 0;
    if (frame)
      o.frame = [&](const std::vector<double>& x, const Cell& c, int64_t step) {
        double cc[12];
        from_cell(c, cc);
        frame(x.data(), cc, step, user);
      };
    o.checkpoint_every = md->checkpoint_every;
    if (md->checkpoint)
      o.checkpoint = [&](const std::vector<double>& x, const std::vector<double>& v, const Cell& c, int64_t step) {
        double cc[12];
        from_cell(c, cc);
        md->checkpoint(x.data(), v.data(), cc, step, md->checkpoint_user);
      };
    o.step_offset = md->step_offset;
    o.respa = md->respa > 1 ? md->respa : 1;
    o.energy = to_eo(eo, threads);
    int k = 0;
    o.progress = [&](const ThermoRow& r) {
      if (k < max_rows) {
        caps_gpu_thermo& t = rows[k];
        std::memset(&t, 0, sizeof t);
        t.step = r.step;
        t.time_ps = r.time_ps;
        t.temperature = r.temperature;
        t.potential = r.potential;
        t.kinetic = r.kinetic;
        t.total = r.total;
        t.conserved = r.conserved;
        t.pressure = r.pressure;
        t.volume = r.volume;
        t.density = r.density;
        t.target_temperature = r.target_temperature;
        for (int c = 0; c < 6; ++c) t.p[c] = r.p[c];
      }
      ++k;
      return true;
    };
    DynamicsReport rep;
    int rc = 0;
    try {
      run_dynamics(s, o, &rep);
    } catch (const DynamicsInterrupted& di) {
      g_err = di.what();
      rc = 1;
    }
    *nrows = k;
    *seconds = rep.seconds;
    *ns_per_day = rep.ns_per_day;
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) {
        st->x[3 * i + c] = s.atoms[size_t(i)].pos[c];
        if (st->v) st->v[3 * i + c] = s.velocities[size_t(i)][c];
      }
    from_cell(s.cell, st->cell);
    return rc;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

void ref_request_stop(int on) { request_stop(on != 0); }

// Evaluator::freeze_pairs at (x0, cell0), then compute at (x1, cell1): forces, terms and pairs().
int ref_freeze_compute(const caps_gpu_ff* p, const caps_gpu_opts* o, const double* x0, const double* cell0, const double* x1, const double* cell1,
                       double* f, caps_gpu_terms* out, int64_t* npairs, int threads) {
  try {
    auto ff = to_ff(p);
    Evaluator ev(*ff, to_eo(o, threads));
    const size_t n3 = 3 * size_t(p->natoms);
    std::vector<double> a(x0, x0 + n3), b(x1, x1 + n3), fv;
    ev.freeze_pairs(a, to_cell(cell0));
    const EnergyTerms t = ev.compute(b, to_cell(cell1), fv);
    std::memcpy(f, fv.data(), n3 * sizeof(double));
    to_terms(t, out);
    *npairs = int64_t(ev.pairs());
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// compute at (x, cell), then pairs().
int ref_pairs(const caps_gpu_ff* p, const caps_gpu_opts* o, const double* x, const double* cell, int64_t* npairs, int threads) {
  try {
    auto ff = to_ff(p);
    Evaluator ev(*ff, to_eo(o, threads));
    std::vector<double> a(x, x + 3 * size_t(p->natoms)), fv;
    ev.compute(a, to_cell(cell), fv);
    *npairs = int64_t(ev.pairs());
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// An evaluator on force field p1 computes at (x, cell); the force field is then changed in place to p2 and reloaded
// (Evaluator::reload, as a bond-exchange move does), and computes again: forces and terms of the second call.
int ref_reload_compute(const caps_gpu_ff* p1, const caps_gpu_ff* p2, const caps_gpu_opts* o, const double* x, const double* cell, double* f,
                       caps_gpu_terms* out, int threads) {
  try {
    auto ff = to_ff(p1);
    Evaluator ev(*ff, to_eo(o, threads));
    const size_t n3 = 3 * size_t(p1->natoms);
    std::vector<double> a(x, x + n3), fv;
    ev.compute(a, to_cell(cell), fv);
    *ff = *to_ff(p2);
    ev.reload();
    const EnergyTerms t = ev.compute(a, to_cell(cell), fv);
    std::memcpy(f, fv.data(), n3 * sizeof(double));
    to_terms(t, out);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// caps::write_trajectory (io_traj.cpp:47) on a Trajectory of nf frames: x [nf][3n], cells [nf][12], steps [nf]; the
// topology's atoms carry ids, mols and types, its title the DCD's second title line.
int ref_write_trajectory(const char* path, int n, const int64_t* ids, const int64_t* mols, const int32_t* types, const char* title, int nf,
                         const double* x, const double* cells, const int64_t* steps, double dt_fs) {
  try {
    Trajectory t;
    t.topology.atoms.resize(size_t(n));
    for (int i = 0; i < n; ++i) {
      Atom& a = t.topology.atoms[size_t(i)];
      a.id = ids[i];
      a.mol = mols[i];
      a.type = types[i];
      a.element = 6;
      for (int k = 0; k < 3; ++k) a.pos[k] = x[3 * size_t(i) + size_t(k)];
    }
    t.topology.title = title ? title : "";
    for (int f = 0; f < nf; ++f) {
      std::vector<Vec3> pos(static_cast<size_t>(n));
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) pos[size_t(i)][k] = x[(size_t(f) * size_t(n) + size_t(i)) * 3 + size_t(k)];
      t.positions.push_back(std::move(pos));
      t.cells.push_back(to_cell(cells + 12 * size_t(f)));
      t.timesteps.push_back(steps[f]);
    }
    if (nf > 0) t.topology.cell = t.cells.front();
    write_trajectory(t, path, dt_fs);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

double ref_ewald_beta(double rc, double rtol) { return ewald_beta(rc, rtol); }

void ref_pme_grid(const double* cell, double beta, double spacing, int order, int* k) {
  const PmeGrid g = pme_grid(to_cell(cell), beta, spacing, order);
  for (int d = 0; d < 3; ++d) k[d] = g.k[d];
}

// The threaded half-spectrum PME of the evaluator (kspace.cpp:80) on given arrays; forces added to f.
double ref_pme(int n, const double* x, const double* q, const double* cell, const int* k, int order, double beta, double* f, double* vir, int threads) {
  std::vector<double> xv(x, x + 3 * size_t(n)), qv(q, q + n), fv(f, f + 3 * size_t(n));
  PmeGrid g;
  for (int d = 0; d < 3; ++d) g.k[d] = k[d];
  g.order = order;
  g.beta = beta;
  ThreadPool pool(threads > 0 ? threads : 1);
  const double e = pme_reciprocal(xv, qv, to_cell(cell), g, fv, vir, pool);
  std::memcpy(f, fv.data(), fv.size() * sizeof(double));
  return e;
}

// The plain Ewald reciprocal sum of the reference (kspace.hpp:28, over |m_d| <= kmax[d]); forces added to f.
double ref_ewald(int n, const double* x, const double* q, const double* cell, const int* kmax, double beta, double* f, double* vir) {
  std::vector<double> xv(x, x + 3 * size_t(n)), qv(q, q + n), fv(f, f + 3 * size_t(n));
  const double e = ewald_reciprocal(xv, qv, to_cell(cell), beta, kmax, fv, vir);
  std::memcpy(f, fv.data(), fv.size() * sizeof(double));
  return e;
}

// Builders: a grown and relaxed atactic polystyrene cell with GAFF (tests/test_nbnxm.cpp:19-34 builds the same kind).
int ref_build_ps_gaff(int chains, int dp, double grow_density, double target_density, uint64_t seed, const char* path) {
  try {
    GrowOptions g;
    g.chains = chains;
    g.dp = dp;
    g.density = grow_density;
    g.seed = seed;
    System c = grow(g);
    RelaxOptions r;
    r.target_density = target_density;
    r.ftol = 1.0;
    relax(c, r);
    const ForceField ff = assign_gaff(c);
    export_system(c, ff, path);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// A Kremer-Grest melt (random-walk chains, not pushed off) with its FENE-WCA force field, in reduced units mapped as
// sigma = 1 Å, eps = kB T at T = 1/kB... the caller picks; here the unmapped reduced model (1 Å, 1 kcal/mol, 1 g/mol).
int ref_build_kg(int chains, int beads, double density, uint64_t seed, const char* path) {
  try {
    KgOptions o;
    o.chains = chains;
    o.beads = beads;
    o.density = density;
    o.seed = seed;
    System s = kremer_grest(o);
    const ForceField ff = kremer_grest_forcefield(s, o);
    export_system(s, ff, path);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// The reference's Tg fits on given points: method 0 fit_bilinear, 1 fit_two_ranges.
int ref_fit_tg(const double* T, const double* y, int n, int method, double glassy_max, double rubbery_min, ref_tg_fit* out) {
  try {
    const std::vector<double> t(T, T + n), v(y, y + n);
    to_fit(method == 1 ? fit_two_ranges(t, v, glassy_max, rubbery_min) : fit_bilinear(t, v), out);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// run_cooling on a System rebuilt from the arrays. opt: t_start, t_end, t_step, ps_per_step, equilibrate_ps,
// average_from, dt, tau_t, tau_p, pressure, compressibility, glassy_max, rubbery_min; iopt: barostat (0 none, 1
// c-rescale), seed, new_velocities, property, fit. points: up to max_points x 5 (T, density, density_err,
// specific volume, potential). The end state is written back to st.
int ref_run_cooling(const caps_gpu_ff* p, const caps_gpu_opts* eo, caps_gpu_state* st, const double* opt, const int64_t* iopt,
                    const int32_t* element, int threads, double* points, int max_points, int* npoints, ref_tg_fit* fit) {
  try {
    auto ff = to_ff(p);
    System s = to_system(p, ff, st, element);
    CoolingOptions o;
    o.field = ff;
    o.energy = to_eo(eo, threads);
    o.t_start = opt[0], o.t_end = opt[1], o.t_step = opt[2], o.ps_per_step = opt[3], o.equilibrate_ps = opt[4];
    o.average_from = opt[5], o.dt = opt[6], o.tau_t = opt[7], o.tau_p = opt[8], o.pressure = opt[9], o.compressibility = opt[10];
    o.glassy_max = opt[11], o.rubbery_min = opt[12];
    o.barostat = iopt[0] == 1 ? Barostat::CRescale : Barostat::None;
    o.seed = uint64_t(iopt[1]);
    o.new_velocities = iopt[2] != 0;
    o.property = int(iopt[3]);
    o.fit = int(iopt[4]);
    const CoolingResult r = run_cooling(s, o);
    *npoints = int(r.points.size());
    for (int k = 0; k < std::min(*npoints, max_points); ++k) {
      const CoolingPoint& q = r.points[size_t(k)];
      double* d = points + 5 * k;
      d[0] = q.temperature, d[1] = q.density, d[2] = q.density_err, d[3] = q.specific_volume, d[4] = q.potential;
    }
    to_fit(r.fit, fit);
    const int n = p->natoms;
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) {
        st->x[3 * i + c] = s.atoms[size_t(i)].pos[c];
        if (st->v) st->v[3 * i + c] = s.velocities[size_t(i)][c];
      }
    from_cell(s.cell, st->cell);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// equilibrate over given stages. ensemble[k]: 0 NVT, 1 NPT, 2 NVE; sd[5k..]: ps, t_start, t_end, pressure, force_cap.
// md: the base dynamics options (dt, thermostat, tau_t, barostat, tau_p, compressibility, seed; energy from eo).
// out[6k..]: ps, temperature, pressure, density, potential, density_end of each stage. The end state goes back to st.
int ref_equilibrate(const caps_gpu_ff* p, const caps_gpu_opts* eo, caps_gpu_state* st, const caps_gpu_md_opts* md, int nstages,
                    const int32_t* ensemble, const double* sd, double thermo_ps, const int32_t* element, int threads, double* out) {
  try {
    auto ff = to_ff(p);
    System s = to_system(p, ff, st, element);
    EquilibrateOptions o;
    for (int k = 0; k < nstages; ++k) {
      Stage g;
      g.label = "stage " + std::to_string(k + 1);
      g.ensemble = ensemble[k] == 1 ? Ensemble::NPT : ensemble[k] == 2 ? Ensemble::NVE : Ensemble::NVT;
      g.ps = sd[5 * k], g.t_start = sd[5 * k + 1], g.t_end = sd[5 * k + 2], g.pressure = sd[5 * k + 3], g.force_cap = sd[5 * k + 4];
      o.stages.push_back(g);
    }
    o.md.field = ff;
    o.md.dt = md->dt;
    const Thermostat th[4] = {Thermostat::None, Thermostat::Bussi, Thermostat::Langevin, Thermostat::NoseHoover};
    o.md.thermostat = th[md->thermostat & 3];
    o.md.tau_t = md->tau_t;
    o.md.barostat = md->barostat == 1 ? Barostat::CRescale : Barostat::None;
    o.md.tau_p = md->tau_p;
    o.md.compressibility = md->compressibility;
    o.md.barostat_every = md->barostat_every;
    o.md.constraints = md->constraints ? ConstraintMode::HBonds : ConstraintMode::None;
    o.md.seed = md->seed;
    o.md.energy = to_eo(eo, threads);
    o.thermo_ps = thermo_ps;
    EquilibrateReport rep;
    equilibrate(s, o, &rep);
    for (size_t k = 0; k < rep.stages.size() && int(k) < nstages; ++k) {
      const StageSummary& q = rep.stages[k];
      double* d = out + 6 * k;
      d[0] = q.ps, d[1] = q.temperature, d[2] = q.pressure, d[3] = q.density, d[4] = q.potential, d[5] = q.density_end;
    }
    const int n = p->natoms;
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) {
        st->x[3 * i + c] = s.atoms[size_t(i)].pos[c];
        if (st->v) st->v[3 * i + c] = s.velocities[size_t(i)][c];
      }
    from_cell(s.cell, st->cell);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// minimise on an evaluator of the arrays' force field. method: 0 SD, 1 CG, 2 L-BFGS, 3 FIRE. fixed: [natoms] or NULL.
// restr: nr x (i, j, r0, k); dihed: nd x (i, j, k, l, phi0, kphi). res: iterations, energy, fmax, evaluations; stopped:
// 0 force, 1 energy, 2 iterations, 3 line search. x is minimised in place.
int ref_minimise(const caps_gpu_ff* p, const caps_gpu_opts* eo, double* x, const double* cell, int method, double ftol, double etol, int max_it,
                 const char* fixed, int nr, const double* restr, int nd, const double* dihed, double* res, int* stopped) {
  try {
    auto ff = to_ff(p);
    RelaxOptions o;
    const Minimiser ms[4] = {Minimiser::SteepestDescent, Minimiser::ConjugateGradient, Minimiser::LBFGS, Minimiser::FIRE};
    o.method = ms[method & 3];
    o.ftol = ftol, o.etol = etol, o.max_iterations = max_it;
    o.energy = to_eo(eo, 1);
    if (fixed) o.fixed.assign(fixed, fixed + p->natoms);
    for (int k = 0; k < nr; ++k) {
      RelaxOptions::Restraint r;
      r.i = uint32_t(restr[4 * k]), r.j = uint32_t(restr[4 * k + 1]), r.r0 = restr[4 * k + 2], r.k = restr[4 * k + 3];
      o.restraints.push_back(r);
    }
    for (int k = 0; k < nd; ++k) {
      RelaxOptions::DihedralRestraint r;
      const double* q = dihed + 6 * k;
      r.i = uint32_t(q[0]), r.j = uint32_t(q[1]), r.k = uint32_t(q[2]), r.l = uint32_t(q[3]), r.phi0 = q[4], r.kphi = q[5];
      o.dihedral_restraints.push_back(r);
    }
    Evaluator ev(*ff, o.energy);
    std::vector<double> xv(x, x + 3 * size_t(p->natoms));
    int nev = 0;
    const RelaxStage st = minimise(ev, xv, to_cell(cell), o, "minimise", &nev);
    std::memcpy(x, xv.data(), xv.size() * sizeof(double));
    res[0] = st.iterations, res[1] = st.energy, res[2] = st.fmax, res[3] = nev;
    *stopped = st.stopped_by == "force" ? 0 : st.stopped_by == "energy" ? 1 : st.stopped_by == "iterations" ? 2 : 3;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// A persistent reference evaluator: the same Evaluator object across calls, so that its pair list keeps the history a
// driver's evaluator has (the order of the pair sums, and so the last bits, follow it).
struct RefEv {
  std::shared_ptr<ForceField> ff;
  std::unique_ptr<Evaluator> ev;
};
void* ref_ev_create(const caps_gpu_ff* p, const caps_gpu_opts* o, int threads) {
  try {
    auto h = std::make_unique<RefEv>();
    h->ff = to_ff(p);
    h->ev = std::make_unique<Evaluator>(*h->ff, to_eo(o, threads));
    return h.release();
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
int ref_ev_set_options(void* h, const caps_gpu_opts* o, int threads) {
  try {
    static_cast<RefEv*>(h)->ev->set_options(to_eo(o, threads));
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ref_ev_compute(void* h, const double* x, const double* cell, double* f, caps_gpu_terms* out) {
  try {
    RefEv* r = static_cast<RefEv*>(h);
    const size_t n3 = 3 * r->ff->atom_type.size();
    std::vector<double> xv(x, x + n3), fv;
    const EnergyTerms t = r->ev->compute(xv, to_cell(cell), fv);
    std::memcpy(f, fv.data(), n3 * sizeof(double));
    to_terms(t, out);
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int ref_ev_list_builds(void* h) { return static_cast<RefEv*>(h)->ev->list_builds(); }
void ref_ev_destroy(void* h) { delete static_cast<RefEv*>(h); }

// relax (relax.cpp:343) with the given force field on a System built from the arrays (check_cell_fit off). opt: method,
// ftol, etol, max_iterations, pushoff, pushoff_ramp_ps, pushoff_cap, pushoff_temperature, pushoff_ramp_segments,
// target_density, compress_step, relax_box, pressure, pressure_tol, box_cycles, box_anisotropic, box axis x, y, z
// (18 numbers); caps: ncaps push-off caps. Out: x and cell in place; res: fmax_initial, fmax_final, density_initial,
// density_final, pressure_final, iterations, evaluations, converged, initial total, final total, stages; per stage (up to
// max_stages) iterations, energy, fmax, density, pressure, stopped_by code in st[6 k..]; names and notes joined by '\n'.
int ref_relax(const caps_gpu_ff* p, const caps_gpu_opts* eo, double* x, double* cell, const double* opt, int ncaps, const double* caps,
              const char* fixed, double* res, int max_stages, double* st, char* names, int names_cap, char* notes, int notes_cap) {
  try {
    auto ff = to_ff(p);
    caps_gpu_state state{x, nullptr, cell, 0};
    System s = to_system(p, ff, &state, nullptr);
    RelaxOptions o;
    const Minimiser ms[4] = {Minimiser::SteepestDescent, Minimiser::ConjugateGradient, Minimiser::LBFGS, Minimiser::FIRE};
    o.method = ms[int(opt[0]) & 3];
    o.ftol = opt[1], o.etol = opt[2], o.max_iterations = int(opt[3]);
    o.check_cell_fit = false;
    o.energy = to_eo(eo, 1);
    o.field = ff;
    o.pushoff = opt[4] != 0;
    o.pushoff_ramp_ps = opt[5], o.pushoff_cap = opt[6], o.pushoff_temperature = opt[7], o.pushoff_ramp_segments = int(opt[8]);
    o.target_density = opt[9], o.compress_step = opt[10];
    o.relax_box = opt[11] != 0;
    o.pressure = opt[12], o.pressure_tol = opt[13], o.box_cycles = int(opt[14]);
    o.box_anisotropic = opt[15] != 0;
    for (int k = 0; k < 3; ++k) o.box_axes[k] = opt[16 + k] != 0;
    o.pushoff_caps.assign(caps, caps + ncaps);
    if (fixed) o.fixed.assign(fixed, fixed + p->natoms);
    RelaxReport rep;
    relax(s, o, &rep);
    for (int i = 0; i < p->natoms; ++i)
      for (int k = 0; k < 3; ++k) x[3 * i + k] = s.atoms[size_t(i)].pos[k];
    from_cell(s.cell, cell);
    res[0] = rep.fmax_initial, res[1] = rep.fmax_final, res[2] = rep.density_initial, res[3] = rep.density_final;
    res[4] = rep.pressure_final, res[5] = rep.iterations, res[6] = rep.evaluations, res[7] = rep.converged ? 1 : 0;
    res[8] = rep.initial.total(), res[9] = rep.final.total(), res[10] = double(rep.stages.size());
    std::string nm, nt;
    for (size_t k = 0; k < rep.stages.size(); ++k) {
      const RelaxStage& r = rep.stages[k];
      nm += r.name + "\n";
      if (int(k) >= max_stages) continue;
      const std::string& b = r.stopped_by;
      st[6 * k] = r.iterations, st[6 * k + 1] = r.energy, st[6 * k + 2] = r.fmax, st[6 * k + 3] = r.density, st[6 * k + 4] = r.pressure;
      st[6 * k + 5] = b == "force" ? 0 : b == "energy" ? 1 : b == "iterations" ? 2 : b == "line search" ? 3 : 4;
    }
    for (const auto& n : rep.notes) nt += n + "\n";
    std::snprintf(names, size_t(names_cap), "%s", nm.c_str());
    std::snprintf(notes, size_t(notes_cap), "%s", nt.c_str());
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // extern "C"
