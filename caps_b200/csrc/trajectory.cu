// Trajectory writers that take frames as a run produces them (caps_gpu_traj_*): the LAMMPS text dump
// (core/src/io_lammps.cpp:585-617), LAMMPS's DCD (core/src/io_binary.cpp:414-462) and GROMACS's TRR
// (core/src/io_traj.cpp:81-107). The reference writes a whole Trajectory held in memory; these write each frame when it
// arrives, so a long run's frames never pile up on the host, and complete what depends on the whole run (DCD's frame
// count and step range) when the file is closed. The bytes are the reference's for the same frames: the same records,
// the same number formats and the same arithmetic for the cell in LAMMPS's form.
// Host code, no device needed.
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "caps_gpu.h"

namespace capsb {
void set_call_error(const std::string& text);   // engine.cu: the text caps_gpu_error(NULL) returns
}

namespace {

struct V3 {
  double x[3];
  double operator[](int k) const { return x[k]; }
};
double dot3(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
V3 cross3(const V3& a, const V3& b) { return {{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}}; }
double norm3(const V3& a) { return std::sqrt(dot3(a, a)); }
V3 scale3(const V3& a, double s) { return {{a[0] * s, a[1] * s, a[2] * s}}; }
V3 add3(const V3& a, const V3& b) { return {{a[0] + b[0], a[1] + b[1], a[2] + b[2]}}; }
V3 sub3(const V3& a, const V3& b) { return {{a[0] - b[0], a[1] - b[1], a[2] - b[2]}}; }

// cell[12] = origin, a, b, c
struct Box {
  V3 o, a, b, c;
  explicit Box(const double* p) : o{{p[0], p[1], p[2]}}, a{{p[3], p[4], p[5]}}, b{{p[6], p[7], p[8]}}, c{{p[9], p[10], p[11]}} {}
  // a cell with a volume (Cell::valid, core/src/system.cpp:14-16)
  bool valid() const { return std::fabs(dot3(a, cross3(b, c))) > 1e-9; }
};

// The cell in LAMMPS's form (a along x, b in the xy plane, c with z > 0) by a proper rotation about the origin, and the
// map of positions with it; a cell already in that form is kept as it is (io_lammps.cpp:70-102).
struct LmpFrame {
  Box cell;
  bool rotated = false;
  V3 ex{{1, 0, 0}}, ey{{0, 1, 0}}, ez{{0, 0, 1}}, origin{{0, 0, 0}};
  explicit LmpFrame(const Box& c) : cell(c), origin(c.o) {
    if (!c.valid()) return;
    const double tol = 1e-10 * std::max({norm3(c.a), norm3(c.b), norm3(c.c), 1.0});
    if (std::fabs(c.a[1]) <= tol && std::fabs(c.a[2]) <= tol && std::fabs(c.b[2]) <= tol && c.a[0] > 0 && c.b[1] > 0 && c.c[2] > 0) return;
    const V3 n = cross3(c.a, c.b);
    rotated = true;
    ex = scale3(c.a, 1.0 / norm3(c.a));
    ez = scale3(n, 1.0 / norm3(n));
    ey = cross3(ez, ex);
    cell.a = {{norm3(c.a), 0, 0}};
    cell.b = {{dot3(c.b, ex), dot3(c.b, ey), 0}};
    cell.c = {{dot3(c.c, ex), dot3(c.c, ey), dot3(c.c, ez)}};
    if (cell.c[2] < 0) {   // c points below the ab plane: move the origin by c and flip c, which spans the same cell
      cell.o = add3(cell.o, cell.c);
      cell.c = scale3(cell.c, -1.0);
    }
  }
  V3 to_frame(const V3& r) const {
    if (!rotated) return r;
    const V3 d = sub3(r, origin);
    return add3(origin, V3{{dot3(d, ex), dot3(d, ey), dot3(d, ez)}});
  }
};

enum class Fmt { Dump, Dcd, Trr };

}  // namespace

struct caps_gpu_traj {
  std::string path;
  Fmt fmt = Fmt::Dump;
  std::FILE* f = nullptr;
  std::vector<char> iobuf;
  int32_t n = 0;
  std::vector<long long> ids, mols;
  std::vector<int> types;
  std::string title;
  double dt_fs = 1.0;
  int64_t frames = 0, first_step = 0, second_step = 0, last_step = 0;
  bool dcd_cells = false;
  std::string err;
  std::vector<float> fbuf;
  std::string text;
  std::vector<std::string> chunks;
  std::vector<unsigned char> bebuf;

  void fail(const std::string& what) {
    if (err.empty()) err = what;
  }
  void put(const void* p, size_t len) {
    if (len && std::fwrite(p, 1, len, f) != len) fail("cannot write " + path + ": " + std::strerror(errno));
  }
  void i32le(int32_t v) { put(&v, 4); }   // DCD: the host's (little-endian) order, as the reference writes it
  void record(const void* p, int32_t len) {
    i32le(len);
    put(p, size_t(len));
    i32le(len);
  }
  // XDR: big-endian 32-bit words
  void i32be(int32_t v) {
    const uint32_t u = uint32_t(v);
    const unsigned char b[4] = {static_cast<unsigned char>(u >> 24), static_cast<unsigned char>(u >> 16), static_cast<unsigned char>(u >> 8),
                                static_cast<unsigned char>(u)};
    put(b, 4);
  }
  void f32be(float x) {
    int32_t v;
    std::memcpy(&v, &x, 4);
    i32be(v);
  }
  void strbe(const char* s) {
    const int32_t len = int32_t(std::strlen(s));
    i32be(len);
    put(s, size_t(len));
    static const char zeros[4] = {0, 0, 0, 0};
    put(zeros, size_t((4 - len % 4) % 4));
  }

  // DCD header (io_binary.cpp:422-448): the control words that depend on the whole run are written as for no frames and
  // completed by finish_dcd
  void dcd_header() {
    char h[84] = {};
    std::memcpy(h, "CORD", 4);
    int32_t ic[20] = {};
    ic[2] = 1;
    const float delta = float(dt_fs / 48.88821);   // the time step in units of 48.88821 fs (the CHARMM convention DCD readers expect)
    std::memcpy(&ic[9], &delta, 4);
    ic[19] = 24;
    std::memcpy(h + 4, ic, 80);
    record(h, 84);
    char ti[4 + 2 * 80];
    const int32_t two = 2;
    std::memcpy(ti, &two, 4);
    std::string l1 = "Created by CAPS", l2 = title.substr(0, 80);
    l1.resize(80, ' ');
    l2.resize(80, ' ');
    std::memcpy(ti + 4, l1.data(), 80);
    std::memcpy(ti + 84, l2.data(), 80);
    record(ti, int32_t(sizeof ti));
    const int32_t na = n;
    record(&na, 4);
  }
  void finish_dcd() {
    // ic[0] frames, ic[1] first step, ic[2] steps between frames, ic[3] last - first, ic[10] unit-cell records; the
    // control words start 8 bytes into the file (record length, "CORD")
    int32_t ic03[4] = {int32_t(frames), frames ? int32_t(first_step) : 0, frames > 1 ? int32_t(std::max<int64_t>(1, second_step - first_step)) : 1,
                       frames ? int32_t(last_step - first_step) : 0};
    const int32_t ic10 = dcd_cells ? 1 : 0;
    if (std::fflush(f) != 0) fail("cannot write " + path + ": " + std::strerror(errno));
    if (std::fseek(f, 8, SEEK_SET) != 0) return fail("cannot complete " + path + ": " + std::strerror(errno));
    put(ic03, sizeof ic03);
    if (std::fseek(f, 8 + 40, SEEK_SET) != 0) return fail("cannot complete " + path + ": " + std::strerror(errno));
    put(&ic10, 4);
  }

  void dcd_frame(const double* x, const Box& c) {
    if (frames == 0) dcd_cells = c.valid();   // the reference's flag is "any frame has a cell"; streamed, the first frame's
    if (dcd_cells) {
      const double la = norm3(c.a), lb = norm3(c.b), lc = norm3(c.c);
      auto cosang = [](const V3& u, const V3& v) {
        const double d = norm3(u) * norm3(v);
        return d > 0 ? dot3(u, v) / d : 0.0;
      };
      const double d[6] = {la, cosang(c.a, c.b), lb, cosang(c.a, c.c), cosang(c.b, c.c), lc};
      record(d, 48);
    }
    fbuf.resize(size_t(n));
    for (int k = 0; k < 3; ++k) {
      for (int32_t i = 0; i < n; ++i) fbuf[size_t(i)] = float(x[3 * size_t(i) + size_t(k)]);
      record(fbuf.data(), int32_t(4 * n));
    }
  }

  // io_lammps.cpp:585-610
  void dump_frame(const double* x, const Box& cell, int64_t step) {
    char b[256];
    const LmpFrame fr(cell);
    const Box& c = fr.cell;
    const bool tri = std::fabs(c.b[0]) + std::fabs(c.c[0]) + std::fabs(c.c[1]) > 0;
    text.clear();
    std::snprintf(b, sizeof b, "ITEM: TIMESTEP\n%lld\nITEM: NUMBER OF ATOMS\n%d\n", static_cast<long long>(step), n);
    text += b;
    const double xlo = c.o[0], ylo = c.o[1], zlo = c.o[2];
    const double xhi = xlo + c.a[0], yhi = ylo + c.b[1], zhi = zlo + c.c[2];
    if (tri) {
      const double xy = c.b[0], xz = c.c[0], yz = c.c[1];
      std::snprintf(b, sizeof b, "ITEM: BOX BOUNDS xy xz yz pp pp pp\n%.6f %.6f %.6f\n%.6f %.6f %.6f\n%.6f %.6f %.6f\n",
                    xlo + std::min({0.0, xy, xz, xy + xz}), xhi + std::max({0.0, xy, xz, xy + xz}), xy, ylo + std::min(0.0, yz),
                    yhi + std::max(0.0, yz), xz, zlo, zhi, yz);
    } else {
      std::snprintf(b, sizeof b, "ITEM: BOX BOUNDS pp pp pp\n%.6f %.6f\n%.6f %.6f\n%.6f %.6f\n", xlo, xhi, ylo, yhi, zlo, zhi);
    }
    text += b;
    text += "ITEM: ATOMS id mol type xu yu zu\n";
    put(text.data(), text.size());
    // the atom lines ("%lld %lld %d %.5f %.5f %.5f\n") by std::to_chars, whose fixed form is printf's to the digit, in
    // chunks formatted on parallel threads for large frames
    const int nt = n >= 16384 ? int(std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency()))) : 1;
    chunks.resize(size_t(nt));
    auto lines = [&](int t) {
      std::string& out = chunks[size_t(t)];
      out.clear();
      const int32_t i0 = int32_t(int64_t(n) * t / nt), i1 = int32_t(int64_t(n) * (t + 1) / nt);
      out.reserve(size_t(i1 - i0) * 48);
      char line[160];
      for (int32_t i = i0; i < i1; ++i) {
        const V3 r = fr.to_frame(V3{{x[3 * size_t(i)], x[3 * size_t(i) + 1], x[3 * size_t(i) + 2]}});
        char* p = line;
        char* const end = line + sizeof line;
        p = std::to_chars(p, p + 24, ids[size_t(i)]).ptr;   // an integer takes at most 20 characters
        *p++ = ' ';
        p = std::to_chars(p, p + 24, mols[size_t(i)]).ptr;
        *p++ = ' ';
        p = std::to_chars(p, p + 24, types[size_t(i)]).ptr;
        bool fits = true;
        for (int d = 0; d < 3 && fits; ++d) {
          *p++ = ' ';
          const auto res = std::to_chars(p, end - 1, r[d], std::chars_format::fixed, 5);
          fits = res.ec == std::errc();
          p = res.ptr;
        }
        if (fits) {
          *p++ = '\n';
          out.append(line, size_t(p - line));
        } else {
          // more digits than the line holds (|x| > 1e100): the reference's own 256-byte line, cut where it cuts it
          char buf[256];
          std::snprintf(buf, sizeof buf, "%lld %lld %d %.5f %.5f %.5f\n", ids[size_t(i)], mols[size_t(i)], types[size_t(i)], r[0], r[1], r[2]);
          out.append(buf);
        }
      }
    };
    std::vector<std::thread> pool;
    pool.reserve(size_t(nt));
    int started = 1;
    try {
      for (; started < nt; ++started) pool.emplace_back(lines, started);
    } catch (const std::exception&) {   // no thread to be had: the rest on this one
    }
    for (int t = started; t < nt; ++t) lines(t);
    lines(0);
    for (auto& th : pool) th.join();
    for (const auto& c : chunks) put(c.data(), c.size());
  }

  // io_traj.cpp:81-107
  void trr_frame(const double* x, const Box& c, int64_t step) {
    const bool box = c.valid();
    const double time_ps = double(step) * dt_fs / 1000.0;
    i32be(1993);
    i32be(13);   // the string's length plus its terminator
    strbe("GMX_trn_file");
    const int32_t sizes[] = {0, 0, box ? 9 * 4 : 0, 0, 0, 0, 0, n * 3 * 4, 0, 0};   // ir e box vir pres top sym x v f
    for (int32_t s : sizes) i32be(s);
    i32be(n);
    i32be(int32_t(step));
    i32be(0);   // nre
    f32be(float(time_ps));
    f32be(0.0f);   // lambda
    if (box)
      for (const V3* v : {&c.a, &c.b, &c.c})
        for (int d = 0; d < 3; ++d) f32be(float((*v)[d] / 10.0));
    // the positions, big-endian, in one write
    bebuf.resize(size_t(n) * 12);
    unsigned char* q = bebuf.data();
    for (size_t k = 0; k < size_t(n) * 3; ++k, q += 4) {
      const float fv = float(x[k] / 10.0);
      uint32_t u;
      std::memcpy(&u, &fv, 4);
      q[0] = static_cast<unsigned char>(u >> 24), q[1] = static_cast<unsigned char>(u >> 16), q[2] = static_cast<unsigned char>(u >> 8),
      q[3] = static_cast<unsigned char>(u);
    }
    put(bebuf.data(), bebuf.size());
  }

  void append(const double* x, const double* cellp, int64_t step) {
    static const double zero_cell[12] = {0};
    const Box c(cellp ? cellp : zero_cell);
    if (frames == 0) first_step = step;
    if (frames == 1) second_step = step;
    last_step = step;
    switch (fmt) {
      case Fmt::Dump: dump_frame(x, c, step); break;
      case Fmt::Dcd: dcd_frame(x, c); break;
      case Fmt::Trr: trr_frame(x, c, step); break;
    }
    ++frames;
  }
};

namespace {
std::string lower_ext(const std::string& path) {
  const auto dot = path.find_last_of('.');
  std::string e = dot == std::string::npos ? "" : path.substr(dot + 1);
  for (auto& ch : e) ch = char(std::tolower(static_cast<unsigned char>(ch)));
  return e;
}
}  // namespace

extern "C" {

caps_gpu_traj* caps_gpu_traj_open(const char* path, int32_t natoms, const int64_t* ids, const int64_t* mols, const int32_t* types, const char* title,
                                  double dt_fs) {
  if (!path || natoms < 0) {
    capsb::set_call_error("caps_gpu_traj_open: a path and natoms >= 0 are needed");
    return nullptr;
  }
  try {
    auto t = std::make_unique<caps_gpu_traj>();
    t->path = path;
    const std::string e = lower_ext(t->path);
    if (e == "lammpstrj" || e == "dump") t->fmt = Fmt::Dump;
    else if (e == "dcd") t->fmt = Fmt::Dcd;
    else if (e == "trr") t->fmt = Fmt::Trr;
    else {
      capsb::set_call_error("trajectory format '" + e + "': the streaming writer takes .lammpstrj, .dump, .dcd or .trr");
      return nullptr;
    }
    t->n = natoms;
    t->ids.resize(size_t(natoms));
    t->mols.resize(size_t(natoms));
    t->types.resize(size_t(natoms));
    for (int32_t i = 0; i < natoms; ++i) {
      t->ids[size_t(i)] = ids ? static_cast<long long>(ids[i]) : i + 1;
      t->mols[size_t(i)] = mols ? static_cast<long long>(mols[i]) : 1;
      t->types[size_t(i)] = types ? types[i] : 1;
    }
    t->title = title ? title : "";
    t->dt_fs = dt_fs;
    t->f = std::fopen(path, t->fmt == Fmt::Dump ? "w" : "wb+");
    if (!t->f) {
      capsb::set_call_error("cannot write " + t->path);
      return nullptr;
    }
    t->iobuf.resize(size_t(1) << 20);
    std::setvbuf(t->f, t->iobuf.data(), _IOFBF, t->iobuf.size());
    if (t->fmt == Fmt::Dcd) t->dcd_header();
    if (!t->err.empty()) {
      std::fclose(t->f);
      capsb::set_call_error(t->err);
      return nullptr;
    }
    return t.release();
  } catch (const std::exception& x) {
    capsb::set_call_error(x.what());
    return nullptr;
  }
}

int32_t caps_gpu_traj_append(caps_gpu_traj* t, const double* x, const double* cell, int64_t step) {
  if (!t || (!x && t->n > 0)) return CAPS_GPU_EINVAL;
  try {
    t->append(x, cell, step);
  } catch (const std::exception& e) {
    t->fail(e.what());
  }
  if (!t->err.empty()) {
    capsb::set_call_error(t->err);
    return CAPS_GPU_EINVAL;
  }
  return CAPS_GPU_OK;
}

void caps_gpu_traj_frame(const double* x, const double* cell, int64_t step, void* user) {
  auto* t = static_cast<caps_gpu_traj*>(user);
  if (!t || !t->err.empty()) return;
  try {
    t->append(x, cell, step);
  } catch (const std::exception& e) {
    t->fail(e.what());
  }
}

int64_t caps_gpu_traj_frames(const caps_gpu_traj* t) { return t ? t->frames : 0; }

int32_t caps_gpu_traj_close(caps_gpu_traj* t) {
  if (!t) return CAPS_GPU_EINVAL;
  std::unique_ptr<caps_gpu_traj> own(t);
  if (t->fmt == Fmt::Dcd && t->err.empty()) t->finish_dcd();
  if (std::fclose(t->f) != 0) t->fail("cannot write " + t->path + ": " + std::strerror(errno));
  if (t->fmt == Fmt::Trr && t->frames == 0 && t->err.empty()) {
    std::remove(t->path.c_str());   // the reference writes no file without frames
    t->fail("no frames to write");
  }
  if (!t->err.empty()) {
    capsb::set_call_error(t->err);
    return CAPS_GPU_EINVAL;
  }
  return CAPS_GPU_OK;
}

}  // extern "C"
