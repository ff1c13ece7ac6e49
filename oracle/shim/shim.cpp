// shim.cpp - TEST INFRASTRUCTURE ONLY.
//
// Single-rank stand-ins for the three external libraries the reference's CPU
// path links (MPI, FFTW3-MPI, LAMMPS), written for this project so that the
// reference's own mpi/SELM*.cpp compile unchanged into oracle/_ref.  Only the
// calls those files make are provided.  FFTs and forces come from the
// oracle's restatement (selm_oracle.c); RanMars restates the published
// Marsaglia-Zaman RANMAR generator with a polar Box-Muller normal.
#include <algorithm>
#include <sys/time.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fftw3-mpi.h"
#include "mpi.h"
#include "shim_lammps_all.h"
#include "../../selm_oracle.h"

// ============================================================ MPI (one rank)
extern "C" {
int MPI_Init(int*, char***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c + 1; return 0; }
int MPI_Comm_free(MPI_Comm*) { return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
double MPI_Wtime(void) {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE) std::memcpy(recvbuf, sendbuf, (size_t)count * (t == MPI_DOUBLE ? 8 : 4));
  return 0;
}
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype st, int, int, void* recvbuf, int, MPI_Datatype,
                 int, int, MPI_Comm, MPI_Status*) {
  std::memmove(recvbuf, sendbuf, (size_t)sendcount * (st == MPI_DOUBLE ? 8 : 4));
  return 0;
}
}

// ============================================================ FFTW-MPI (one rank)
struct shim_fftw_plan_s {
  int kind;  // 0: r2c transposed-out, 1: c2r transposed-in, 2: many c2r transposed-in
  int n0, n1, n2, howmany;
  double* rbuf;
  double* cbuf;  // interleaved re, im
};

extern "C" {
double* fftw_alloc_real(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
void fftw_free(void* p) { free(p); }
void fftw_mpi_init(void) {}

ptrdiff_t fftw_mpi_local_size_many_transposed(int rnk, const ptrdiff_t* n, ptrdiff_t howmany, ptrdiff_t, ptrdiff_t,
                                              MPI_Comm, ptrdiff_t* local_n0, ptrdiff_t* local_0_start,
                                              ptrdiff_t* local_n1, ptrdiff_t* local_1_start) {
  ptrdiff_t tot = howmany;
  for (int i = 0; i < rnk; i++) tot *= n[i];
  *local_n0 = n[0];
  *local_0_start = 0;
  *local_n1 = n[1];
  *local_1_start = 0;
  return tot;
}

static fftw_plan mk(int kind, ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, int howmany, double* r, double* c,
                    unsigned flags) {
  const unsigned need = (kind == 0) ? FFTW_MPI_TRANSPOSED_OUT : FFTW_MPI_TRANSPOSED_IN;
  if (!(flags & need)) {
    fprintf(stderr, "fftw shim: only the transposed layouts of the reference are provided\n");
    abort();
  }
  fftw_plan p = new shim_fftw_plan_s;
  p->kind = kind;
  p->n0 = (int)n0;
  p->n1 = (int)n1;
  p->n2 = (int)n2;
  p->howmany = howmany;
  p->rbuf = r;
  p->cbuf = c;
  return p;
}

fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double* in, fftw_complex* out, MPI_Comm,
                                   unsigned flags) {
  return mk(0, n0, n1, n2, 1, in, (double*)out, flags);
}
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex* in, double* out, MPI_Comm,
                                   unsigned flags) {
  return mk(1, n0, n1, n2, 1, out, (double*)in, flags);
}
fftw_plan fftw_mpi_plan_many_dft_c2r(int rnk, const ptrdiff_t* n, ptrdiff_t howmany, ptrdiff_t, ptrdiff_t,
                                     fftw_complex* in, double* out, MPI_Comm, unsigned flags) {
  if (rnk != 3) abort();
  return mk(2, n[0], n[1], n[2], (int)howmany, out, (double*)in, flags);
}

void fftw_execute(const fftw_plan p) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, nh = n2 / 2 + 1, H = p->howmany;
  const size_t nr = (size_t)n0 * n1 * n2, nc = (size_t)n0 * n1 * nh;
  std::vector<double> tr(nr), tc(2 * nc);
  if (p->kind == 0) {
    for (int k = 0; k < n0; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < n2; i++) tr[((size_t)k * n1 + j) * n2 + i] = p->rbuf[((size_t)k * n1 + j) * 2 * nh + i];
    orc_fft3_r2c(n2, n1, n0, tr.data(), tc.data());
    for (int k = 0; k < n0; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < nh; i++) {
          const size_t s = ((size_t)k * n1 + j) * nh + i, d = ((size_t)j * n0 + k) * nh + i;
          p->cbuf[2 * d] = tc[2 * s];
          p->cbuf[2 * d + 1] = tc[2 * s + 1];
        }
    return;
  }
  // the reference runs these in place (input and output share the buffer):
  // every field's input is gathered before any output is written
  std::vector<double> tca(2 * nc * H);
  for (int d = 0; d < H; d++)
    for (int k = 0; k < n0; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < nh; i++) {
          const size_t t = ((size_t)k * n1 + j) * nh + i, s = (((size_t)j * n0 + k) * nh + i) * H + d;
          tca[2 * (d * nc + t)] = p->cbuf[2 * s];
          tca[2 * (d * nc + t) + 1] = p->cbuf[2 * s + 1];
        }
  for (int d = 0; d < H; d++) {
    std::copy(tca.begin() + 2 * d * nc, tca.begin() + 2 * (d + 1) * nc, tc.begin());
    orc_fft3_c2r(n2, n1, n0, tc.data(), tr.data());
    for (int k = 0; k < n0; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < n2; i++)
          p->rbuf[(((size_t)k * n1 + j) * 2 * nh + i) * H + d] = tr[((size_t)k * n1 + j) * n2 + i];
  }
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
}

// ============================================================ LAMMPS subset
namespace LAMMPS_NS {

struct ShimModel {
  std::map<std::string, std::string> vars;
  std::string atom_style = "atomic";
  int ntypes = 0, nbondtypes = 0, nangletypes = 0;
  std::vector<double> mass;  // [ntypes+1]
  std::vector<double> xs, vs, fs;
  std::vector<double*> xp, vp, fp;
  std::vector<int> type;
  std::vector<int> bonds, angles;  // (type, i, j) / (type, i, j, k), 0-based local indices
  int bond_style = 0, angle_style = 0, pair_style = 0, pair_shift = 0;
  std::vector<double> bond_coeff, angle_coeff, pair_coeff;
  double pair_rc_global = 0.0;
  double special[4] = {1.0, 0.0, 0.0, 0.0};
  double body[3] = {0.0, 0.0, 0.0};  // fix addforce
  double lo = 0, hi = 0;
};

static std::vector<std::string> split(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> out;
  std::string w;
  while (is >> w) out.push_back(w);
  return out;
}

static std::string strip_comment(std::string line) {
  const size_t p = line.find('#');
  if (p != std::string::npos) line = line.substr(0, p);
  return line;
}

static void ensure_types(ShimModel* m) {
  m->mass.resize(m->ntypes + 1, 0.0);
  m->pair_coeff.resize(3 * (size_t)(m->ntypes + 1) * (m->ntypes + 1), 0.0);
  m->bond_coeff.resize(4 * (size_t)(m->nbondtypes + 1), 0.0);
  m->angle_coeff.resize(2 * (size_t)(m->nangletypes + 1), 0.0);
}

static void type_range(const std::string& s, int n, int& lo, int& hi) {
  if (s == "*") {
    lo = 1;
    hi = n;
  } else {
    lo = hi = std::stoi(s);
  }
}

static void read_data(LAMMPS* lmp, const std::string& path) {
  ShimModel* m = lmp->model;
  std::ifstream in(path);
  if (!in) throw std::runtime_error("shim: cannot open data file " + path);
  std::string line;
  std::getline(in, line);  // title
  int natoms = 0, nbonds = 0, nangles = 0;
  std::string section;
  std::map<long, int> id2idx;
  std::vector<std::string> lines;
  while (std::getline(in, line)) lines.push_back(line);
  size_t li = 0;
  // header
  for (; li < lines.size(); li++) {
    std::vector<std::string> w = split(strip_comment(lines[li]));
    if (w.empty()) continue;
    if (w.size() == 2 && w[1] == "atoms") natoms = std::stoi(w[0]);
    else if (w.size() == 2 && w[1] == "bonds") nbonds = std::stoi(w[0]);
    else if (w.size() == 2 && w[1] == "angles") nangles = std::stoi(w[0]);
    else if (w.size() == 3 && w[1] == "atom" && w[2] == "types") m->ntypes = std::stoi(w[0]);
    else if (w.size() == 3 && w[1] == "bond" && w[2] == "types") m->nbondtypes = std::stoi(w[0]);
    else if (w.size() == 3 && w[1] == "angle" && w[2] == "types") m->nangletypes = std::stoi(w[0]);
    else if (w.size() == 4 && w[2] == "xlo") {
      m->lo = std::stod(w[0]);
      m->hi = std::stod(w[1]);
    } else if (w.size() >= 2 && (w[2 % w.size()] == "ylo" || w[2 % w.size()] == "zlo")) {
    } else if (std::isalpha((unsigned char)w[0][0])) break;
  }
  ensure_types(m);
  m->xs.assign(3 * (size_t)natoms, 0.0);
  m->vs.assign(3 * (size_t)natoms, 0.0);
  m->fs.assign(3 * (size_t)natoms, 0.0);
  m->type.assign(natoms, 1);
  int na = 0;
  std::vector<long> vel_ids;
  std::vector<std::vector<double>> vel_vals;
  std::vector<std::vector<long>> bond_rows, angle_rows;
  for (; li < lines.size(); li++) try {
    const std::string raw = strip_comment(lines[li]);
    std::vector<std::string> w = split(raw);
    if (w.empty()) continue;
    if (std::isalpha((unsigned char)w[0][0])) {
      section = w[0];
      if (w.size() > 1 && w[0] != "Atoms") section += " " + w[1];
      continue;
    }
    if (section == "Masses") {
      m->mass[std::stoi(w[0])] = std::stod(w[1]);
    } else if (section == "Atoms") {
      const bool mol = (m->atom_style != "atomic");
      const long id = std::stol(w[0]);
      const int t = std::stoi(w[mol ? 2 : 1]);
      const int o = mol ? 3 : 2;
      id2idx[id] = na;
      m->type[na] = t;
      for (int d = 0; d < 3; d++) m->xs[3 * na + d] = std::stod(w[o + d]);
      na++;
    } else if (section == "Velocities") {
      vel_ids.push_back(std::stol(w[0]));
      vel_vals.push_back({std::stod(w[1]), std::stod(w[2]), std::stod(w[3])});
    } else if (section == "Bonds") {
      bond_rows.push_back({std::stol(w[1]), std::stol(w[2]), std::stol(w[3])});
    } else if (section == "Angles") {
      angle_rows.push_back({std::stol(w[1]), std::stol(w[2]), std::stol(w[3]), std::stol(w[4])});
    }
  } catch (const std::exception& e) {
    throw std::runtime_error("shim: cannot parse data line '" + lines[li] + "' (" + e.what() + ")");
  }
  if (na != natoms) throw std::runtime_error("shim: atom count mismatch in data file");
  for (size_t q = 0; q < vel_ids.size(); q++)
    for (int d = 0; d < 3; d++) m->vs[3 * id2idx.at(vel_ids[q]) + d] = vel_vals[q][d];
  for (auto& r : bond_rows) {
    m->bonds.push_back((int)r[0]);
    m->bonds.push_back(id2idx.at(r[1]));
    m->bonds.push_back(id2idx.at(r[2]));
  }
  for (auto& r : angle_rows) {
    m->angles.push_back((int)r[0]);
    m->angles.push_back(id2idx.at(r[1]));
    m->angles.push_back(id2idx.at(r[2]));
    m->angles.push_back(id2idx.at(r[3]));
  }
  (void)nbonds;
  (void)nangles;
  m->xp.resize(natoms);
  m->vp.resize(natoms);
  m->fp.resize(natoms);
  for (int i = 0; i < natoms; i++) {
    m->xp[i] = &m->xs[3 * (size_t)i];
    m->vp[i] = &m->vs[3 * (size_t)i];
    m->fp[i] = &m->fs[3 * (size_t)i];
  }
  Atom* a = lmp->atom;
  a->nlocal = natoms;
  a->x = m->xp.data();
  a->v = m->vp.data();
  a->f = m->fp.data();
  a->type = m->type.data();
  a->mass = m->mass.data();
  for (int d = 0; d < 3; d++) {
    lmp->domain->boxlo[d] = m->lo;
    lmp->domain->boxhi[d] = m->hi;
  }
}

static std::string substitute(const std::string& s, const std::map<std::string, std::string>& vars) {
  std::string out;
  for (size_t i = 0; i < s.size(); i++) {
    if (s[i] == '$' && i + 1 < s.size() && s[i + 1] == '{') {
      const size_t e = s.find('}', i);
      const std::string k = s.substr(i + 2, e - i - 2);
      auto it = vars.find(k);
      out += (it != vars.end()) ? it->second : "";
      i = e;
    } else {
      out += s[i];
    }
  }
  return out;
}

void Input::file(const char* path) {
  ShimModel* m = lmp->model;
  std::ifstream in(path);
  if (!in) throw std::runtime_error(std::string("shim: cannot open ") + path);
  std::string line;
  while (std::getline(in, line)) try {
    std::vector<std::string> w = split(substitute(strip_comment(line), m->vars));
    if (w.empty()) continue;
    const std::string& c = w[0];
    if (c == "variable" && w.size() >= 4) m->vars[w[1]] = w[3];
    else if (c == "atom_style") m->atom_style = w[1];
    else if (c == "read_data") read_data(lmp, w[1]);
    else if (c == "timestep") lmp->update->dt = std::stod(w[1]);
    else if (c == "mass") {
      ensure_types(m);
      m->mass[std::stoi(w[1])] = std::stod(w[2]);
    } else if (c == "bond_style") m->bond_style = (w[1] == "harmonic") ? 1 : (w[1] == "fene") ? 2 : 0;
    else if (c == "bond_coeff") {
      ensure_types(m);
      const int t = std::stoi(w[1]);
      for (size_t q = 2; q < w.size() && q < 6; q++) m->bond_coeff[4 * t + q - 2] = std::stod(w[q]);
    } else if (c == "angle_style") m->angle_style = (w[1] == "harmonic") ? 1 : 0;
    else if (c == "angle_coeff") {
      ensure_types(m);
      const int t = std::stoi(w[1]);
      m->angle_coeff[2 * t] = std::stod(w[2]);
      m->angle_coeff[2 * t + 1] = std::stod(w[3]);
    } else if (c == "pair_style") {
      m->pair_style = (w[1] == "lj/cut") ? 1 : 0;
      if (w.size() > 2) m->pair_rc_global = std::stod(w[2]);
    } else if (c == "pair_coeff") {
      ensure_types(m);
      int a0, a1, b0, b1;
      type_range(w[1], m->ntypes, a0, a1);
      type_range(w[2], m->ntypes, b0, b1);
      const double eps = std::stod(w[3]), sig = std::stod(w[4]);
      const double rc = (w.size() > 5) ? std::stod(w[5]) : m->pair_rc_global;
      const int nt1 = m->ntypes + 1;
      for (int i = a0; i <= a1; i++)
        for (int j = b0; j <= b1; j++) {
          for (int q = 0; q < 2; q++) {
            const int ii = q ? j : i, jj = q ? i : j;
            double* pc = &m->pair_coeff[3 * ((size_t)ii * nt1 + jj)];
            pc[0] = eps;
            pc[1] = sig;
            pc[2] = rc;
          }
        }
    } else if (c == "pair_modify") {
      for (size_t q = 1; q + 1 < w.size(); q++)
        if (w[q] == "shift") m->pair_shift = (w[q + 1] == "yes");
    } else if (c == "special_bonds") {
      if (w.size() >= 2 && w[1] == "fene") {
        m->special[1] = 0.0;
        m->special[2] = 1.0;
        m->special[3] = 1.0;
      } else if (w.size() >= 5 && (w[1] == "lj" || w[1] == "lj/coul")) {
        for (int q = 0; q < 3; q++) m->special[q + 1] = std::stod(w[2 + q]);
      }
    }
    else if (c == "fix" && w.size() >= 7 && w[3] == "addforce") {
      for (int q = 0; q < 3; q++) m->body[q] = std::stod(w[4 + q]);
    }
    // units, boundary, log, neighbor, neigh_modify, thermo*, dump, other fixes, run: no effect on the step
  } catch (const std::exception& e) {
    throw std::runtime_error("shim: cannot parse script line '" + line + "' (" + e.what() + ")");
  }
}

LAMMPS::LAMMPS(int, char**, MPI_Comm) {
  model = new ShimModel();
  input = new Input(this);
  update = new Update();
  update->integrate = new Integrate(this);
  atom = new Atom();
  domain = new Domain();
  output = new Output();
}

LAMMPS::~LAMMPS() {
  delete update->integrate;
  delete input;
  delete update;
  delete atom;
  delete domain;
  delete output;
  delete model;
}

void LAMMPS::init() {}

static void compute(LAMMPS* lmp) {
  ShimModel* m = lmp->model;
  const int n = lmp->atom->nlocal;
  // periodic remap of positions (Domain::pbc for a periodic box)
  const double L = m->hi - m->lo;
  for (int i = 0; i < 3 * n; i++) {
    double& x = m->xs[i];
    if (x < m->lo) x += L;
    if (x >= m->hi) {
      x -= L;
      if (x < m->lo) x = m->lo;
    }
  }
  orc_ff ff{};
  ff.natoms = n;
  ff.ntypes = m->ntypes;
  ff.type = m->type.data();
  ff.nbonds = (int)m->bonds.size() / 3;
  ff.bond = m->bonds.data();
  ff.bond_style = m->bond_style;
  ff.bond_coeff = m->bond_coeff.data();
  ff.nangles = (int)m->angles.size() / 4;
  ff.angle = m->angles.data();
  ff.angle_style = m->angle_style;
  ff.angle_coeff = m->angle_coeff.data();
  ff.pair_style = m->pair_style;
  ff.pair_coeff = m->pair_coeff.data();
  ff.pair_shift = m->pair_shift;
  for (int q = 0; q < 4; q++) ff.special_lj[q] = m->special[q];
  for (int q = 0; q < 3; q++) ff.body_force[q] = m->body[q];
  ff.lo = m->lo;
  ff.hi = m->hi;
  orc_forces(&ff, m->xs.data(), m->fs.data());
}

void Integrate::setup(int) { compute(lmp); }
void Integrate::setup_minimal(int) { compute(lmp); }

// ---------------------------------------------------------------- RANMAR
RanMars::RanMars(LAMMPS*, int seed) {
  if (seed <= 0 || seed > 900000000) throw std::runtime_error("shim: invalid seed for RanMars");
  save = 0;
  second = 0.0;
  const int ij = (seed - 1) / 30082, kl = (seed - 1) - 30082 * ij;
  int i = (ij / 177) % 177 + 2, j = ij % 177 + 2, k = (kl / 169) % 178 + 1, l = kl % 169;
  for (int ii = 1; ii <= 97; ii++) {
    double s = 0.0, t = 0.5;
    for (int jj = 1; jj <= 24; jj++) {
      const int mm = ((i * j) % 179) * k % 179;
      i = j;
      j = k;
      k = mm;
      l = (53 * l + 1) % 169;
      if ((l * mm) % 64 >= 32) s += t;
      t *= 0.5;
    }
    u[ii] = s;
  }
  c = 362436.0 / 16777216.0;
  cd = 7654321.0 / 16777216.0;
  cm = 16777213.0 / 16777216.0;
  i97 = 97;
  j97 = 33;
  uniform();
}

double RanMars::uniform() {
  double uni = u[i97] - u[j97];
  if (uni < 0.0) uni += 1.0;
  u[i97] = uni;
  if (--i97 == 0) i97 = 97;
  if (--j97 == 0) j97 = 97;
  c -= cd;
  if (c < 0.0) c += cm;
  uni -= c;
  if (uni < 0.0) uni += 1.0;
  return uni;
}

double RanMars::gaussian() {
  if (save) {
    save = 0;
    return second;
  }
  double v1, v2, rsq;
  do {
    v1 = 2.0 * uniform() - 1.0;
    v2 = 2.0 * uniform() - 1.0;
    rsq = v1 * v1 + v2 * v2;
  } while (rsq >= 1.0 || rsq == 0.0);
  const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
  second = v1 * fac;
  save = 1;
  return v2 * fac;
}

}  // namespace LAMMPS_NS
