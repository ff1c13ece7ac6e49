// selm_input.cpp - reading a reference case directory.
//
// A case directory holds Model.SELM (parsed with the reference's ParmParse
// semantics, cuda/SELM_ParmParse.cuh:19-101: "key value # comment", last
// occurrence wins, required keys via get, optional via query) and
// Model.LAMMPS_script, which the reference hands to an embedded LAMMPS
// (cuda/SELM_Lagrangian_LAMMPS.cu:21-28).  Of that script the subset the
// reference's cases use is read here: variable, atom_style, read_data,
// timestep, mass, bond_style/bond_coeff (harmonic, fene), angle_style/
// angle_coeff (harmonic), pair_style/pair_coeff (lj/cut), special_bonds,
// fix addforce.  Commands that do not change the step (units, boundary, log,
// neighbor, neigh_modify, thermo*, other dumps and fixes) are accepted and
// ignored; a "dump ... dcd N file" is recorded for the selm_b200 executable.
// Keys the reference does not know (form, integrator, noise_mode) select this
// library's forms and are ignored by the reference.
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "selm_engine.h"

namespace {

struct ParmParse {
  std::map<std::string, std::string> data;
  bool load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
      const size_t c = line.find('#');
      if (c != std::string::npos) line = line.substr(0, c);
      std::istringstream is(line);
      std::string key;
      if (!(is >> key)) continue;
      std::string value;
      std::getline(is, value);
      data[key] = value;
    }
    return true;
  }
  template <typename T> void get(const std::string& k, T& v) const {
    auto it = data.find(k);
    if (it == data.end()) throw std::runtime_error("Key not found: " + k);
    std::istringstream is(it->second);
    is >> v;
  }
  // returns true when the key is present (the reference's query returns 0 then)
  template <typename T> bool query(const std::string& k, T& v) const {
    auto it = data.find(k);
    if (it == data.end()) return false;
    std::istringstream is(it->second);
    is >> v;
    return true;
  }
  void get3(const std::string& k, int v[3]) const {
    auto it = data.find(k);
    if (it == data.end()) throw std::runtime_error("Key not found: " + k);
    std::istringstream is(it->second);
    for (int i = 0; i < 3; i++)
      if (!(is >> v[i])) throw std::runtime_error("Not enough data to fill the array for key: " + k);
  }
};

std::vector<std::string> words(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> w;
  std::string t;
  while (is >> t) w.push_back(t);
  return w;
}

std::string no_comment(std::string s) {
  const size_t c = s.find('#');
  return c == std::string::npos ? s : s.substr(0, c);
}

struct Model {
  std::map<std::string, std::string> vars;
  std::string atom_style = "atomic";
  double dt = 1.0;  // LAMMPS "real" default timestep is 1 fs
  double lo = 0, hi = 0;
  int ntypes = 0, nbondtypes = 0, nangletypes = 0;
  std::vector<double> mass;
  std::vector<double> x, v;
  std::vector<int> type, bonds, angles;
  int bond_style = 0, angle_style = 0, pair_style = 0;
  std::vector<double> bond_coeff, angle_coeff, pair_coeff;
  double rc_global = 0;
  double special[3] = {0, 0, 0};
  double body[3] = {0, 0, 0};
  int dump_every = 0;  // dump ID group dcd N file
  std::string dump_file;
  void size_tables() {
    mass.resize(ntypes + 1, 0.0);
    bond_coeff.resize(4 * (size_t)(nbondtypes + 1), 0.0);
    angle_coeff.resize(2 * (size_t)(nangletypes + 1), 0.0);
    pair_coeff.resize(3 * (size_t)(ntypes + 1) * (ntypes + 1), 0.0);
  }
};

std::string subst(const std::string& s, const std::map<std::string, std::string>& vars) {
  std::string out;
  for (size_t i = 0; i < s.size(); i++) {
    if (s[i] == '$' && i + 1 < s.size() && s[i + 1] == '{') {
      const size_t e = s.find('}', i);
      if (e == std::string::npos) throw std::runtime_error("unterminated ${");
      auto it = vars.find(s.substr(i + 2, e - i - 2));
      out += it == vars.end() ? "" : it->second;
      i = e;
    } else {
      out += s[i];
    }
  }
  return out;
}

void read_data(Model& m, const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open data file " + path);
  std::vector<std::string> lines;
  std::string line;
  std::getline(f, line);  // title
  while (std::getline(f, line)) lines.push_back(no_comment(line));
  size_t i = 0;
  int natoms = 0;
  for (; i < lines.size(); i++) {
    auto w = words(lines[i]);
    if (w.empty()) continue;
    if (std::isalpha((unsigned char)w[0][0])) break;
    if (w.size() == 2 && w[1] == "atoms") natoms = std::stoi(w[0]);
    else if (w.size() == 3 && w[1] == "atom" && w[2] == "types") m.ntypes = std::stoi(w[0]);
    else if (w.size() == 3 && w[1] == "bond" && w[2] == "types") m.nbondtypes = std::stoi(w[0]);
    else if (w.size() == 3 && w[1] == "angle" && w[2] == "types") m.nangletypes = std::stoi(w[0]);
    else if (w.size() == 4 && w[2] == "xlo") {
      m.lo = std::stod(w[0]);
      m.hi = std::stod(w[1]);
    }
  }
  m.size_tables();
  m.x.assign(3 * (size_t)natoms, 0.0);
  m.v.assign(3 * (size_t)natoms, 0.0);
  m.type.assign(natoms, 1);
  std::map<long, int> id2;
  std::vector<std::vector<double>> vel;
  std::vector<long> vel_id;
  std::vector<std::vector<long>> b, a;
  std::string sec;
  int na = 0;
  for (; i < lines.size(); i++) {
    auto w = words(lines[i]);
    if (w.empty()) continue;
    if (std::isalpha((unsigned char)w[0][0])) {
      sec = w[0];
      if (w.size() > 1) sec += " " + w[1];
      if (w[0] == "Atoms") sec = "Atoms";
      continue;
    }
    if (sec == "Masses") m.mass.at(std::stoi(w[0])) = std::stod(w.at(1));
    else if (sec == "Atoms") {
      const bool mol = m.atom_style != "atomic";
      if (na >= natoms) throw std::runtime_error("more atoms than declared");
      id2[std::stol(w[0])] = na;
      m.type[na] = std::stoi(w.at(mol ? 2 : 1));
      for (int d = 0; d < 3; d++) m.x[3 * na + d] = std::stod(w.at((mol ? 3 : 2) + d));
      na++;
    } else if (sec == "Velocities") {
      vel_id.push_back(std::stol(w[0]));
      vel.push_back({std::stod(w.at(1)), std::stod(w.at(2)), std::stod(w.at(3))});
    } else if (sec == "Bonds") {
      b.push_back({std::stol(w.at(1)), std::stol(w.at(2)), std::stol(w.at(3))});
    } else if (sec == "Angles") {
      a.push_back({std::stol(w.at(1)), std::stol(w.at(2)), std::stol(w.at(3)), std::stol(w.at(4))});
    }
  }
  if (na != natoms) throw std::runtime_error("atom count differs from the header");
  for (size_t q = 0; q < vel.size(); q++)
    for (int d = 0; d < 3; d++) m.v[3 * id2.at(vel_id[q]) + d] = vel[q][d];
  for (auto& r : b) {
    m.bonds.push_back((int)r[0]);
    m.bonds.push_back(id2.at(r[1]));
    m.bonds.push_back(id2.at(r[2]));
  }
  for (auto& r : a) {
    m.angles.push_back((int)r[0]);
    m.angles.push_back(id2.at(r[1]));
    m.angles.push_back(id2.at(r[2]));
    m.angles.push_back(id2.at(r[3]));
  }
}

void read_script(Model& m, const std::string& dir, const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::string line;
  while (std::getline(f, line)) {
    auto w = words(subst(no_comment(line), m.vars));
    if (w.empty()) continue;
    const std::string& c = w[0];
    if (c == "variable" && w.size() >= 4) m.vars[w[1]] = w[3];
    else if (c == "atom_style") m.atom_style = w.at(1);
    else if (c == "read_data") {
      const std::string p = w.at(1);
      read_data(m, p.size() && p[0] == '/' ? p : dir + "/" + p);
    } else if (c == "timestep") m.dt = std::stod(w.at(1));
    else if (c == "dump" && w.size() >= 6 && w[3] == "dcd") {
      m.dump_every = std::stoi(w[4]);
      m.dump_file = w[5];
    }
    else if (c == "mass") {
      m.size_tables();
      m.mass.at(std::stoi(w.at(1))) = std::stod(w.at(2));
    } else if (c == "bond_style") {
      if (w.at(1) == "harmonic") m.bond_style = SELM_BOND_HARMONIC;
      else if (w[1] == "fene") m.bond_style = SELM_BOND_FENE;
      else throw std::runtime_error("unsupported bond_style " + w[1]);
    } else if (c == "bond_coeff") {
      m.size_tables();
      const int t = std::stoi(w.at(1));
      const size_t nval = (m.bond_style == SELM_BOND_FENE) ? 4 : 2;
      for (size_t q = 0; q < nval; q++) m.bond_coeff.at(4 * t + q) = std::stod(w.at(2 + q));
    } else if (c == "angle_style") {
      if (w.at(1) == "harmonic") m.angle_style = SELM_ANGLE_HARMONIC;
      else throw std::runtime_error("unsupported angle_style " + w[1]);
    } else if (c == "angle_coeff") {
      m.size_tables();
      const int t = std::stoi(w.at(1));
      m.angle_coeff.at(2 * t) = std::stod(w.at(2));
      m.angle_coeff.at(2 * t + 1) = std::stod(w.at(3));
    } else if (c == "pair_style") {
      if (w.at(1) != "lj/cut") throw std::runtime_error("unsupported pair_style " + w[1]);
      m.pair_style = SELM_PAIR_LJCUT;
      if (w.size() > 2) m.rc_global = std::stod(w[2]);
    } else if (c == "pair_coeff") {
      m.size_tables();
      auto range = [&](const std::string& s, int& a, int& b) {
        if (s == "*") {
          a = 1;
          b = m.ntypes;
        } else {
          a = b = std::stoi(s);
        }
      };
      int a0, a1, b0, b1;
      range(w.at(1), a0, a1);
      range(w.at(2), b0, b1);
      const double eps = std::stod(w.at(3)), sig = std::stod(w.at(4));
      const double rc = w.size() > 5 ? std::stod(w[5]) : m.rc_global;
      const int nt1 = m.ntypes + 1;
      for (int i = a0; i <= a1; i++)
        for (int j = b0; j <= b1; j++)
          for (int s = 0; s < 2; s++) {
            const int ii = s ? j : i, jj = s ? i : j;
            double* pc = &m.pair_coeff.at(3 * ((size_t)ii * nt1 + jj));
            pc[0] = eps;
            pc[1] = sig;
            pc[2] = rc;
          }
    } else if (c == "special_bonds") {
      if (w.size() >= 2 && w[1] == "fene") {
        m.special[0] = 0.0;
        m.special[1] = 1.0;
        m.special[2] = 1.0;
      } else if (w.size() >= 5 && (w[1] == "lj" || w[1] == "lj/coul")) {
        for (int q = 0; q < 3; q++) m.special[q] = std::stod(w[2 + q]);
      }
    } else if (c == "fix" && w.size() >= 7 && w[3] == "addforce") {
      for (int q = 0; q < 3; q++) m.body[q] = std::stod(w[4 + q]);
    }
  }
}

}  // namespace

int selm_case_create(const char* case_dir, selm_sim** out) {
  if (!out || !case_dir) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  *out = nullptr;
  const std::string dir(case_dir);
  ParmParse pp;
  if (!pp.load(dir + "/Model.SELM")) return selm_fail(SELM_ERR_IO, "cannot open " + dir + "/Model.SELM");
  selm_params prm{};
  Model m;
  int nsteps = 0;
  try {
    std::string lt, et;
    pp.get("rho", prm.rho);
    pp.get("T", prm.T);
    pp.get("mu", prm.mu);
    pp.get("nsteps", nsteps);
    pp.get("KB", prm.KB);
    pp.get("LagrangianType", lt);
    pp.get("EulerianType", et);
    if (lt != "Lagrangian_LAMMPS") return selm_fail(SELM_ERR_IO, "LagrangianType must be Lagrangian_LAMMPS");
    if (et != "Eulerian_Period") return selm_fail(SELM_ERR_IO, "EulerianType must be Eulerian_Period");
    int flag = 0;
    pp.query("flagStochasticDriving", flag);
    prm.flag_stochastic = flag;
    long long seed = 123456;  // cuda/SELM.cuh:14
    pp.query("SELM_Seed", seed);
    prm.seed = (unsigned long long)seed;
    pp.get3("numMeshPtsPerDir", prm.num_mesh_pts);
    std::string form = "plain64", integ = "inertial", noise = "ref_compat";
    pp.query("form", form);
    pp.query("integrator", integ);
    pp.query("noise_mode", noise);
    prm.form = form == "fused32" ? SELM_FORM_FUSED32 : form == "fused64" ? SELM_FORM_FUSED64 : SELM_FORM_PLAIN64;
    prm.integrator = integ == "quasi_steady" ? SELM_INTEGRATOR_QUASI_STEADY : SELM_INTEGRATOR_INERTIAL;
    prm.noise_mode = noise == "exact" ? SELM_NOISE_EXACT : SELM_NOISE_REF_COMPAT;
    read_script(m, dir, dir + "/Model.LAMMPS_script");
  } catch (const std::exception& e) {
    return selm_fail(SELM_ERR_IO, e.what());
  }
  prm.dt = m.dt;
  prm.box_lo = m.lo;
  prm.box_hi = m.hi;
  selm_sim* s = nullptr;
  int rc = selm_create(&prm, &s);
  if (rc) return rc;
  const int M = (int)m.type.size();
  std::vector<double> mass(M);
  for (int i = 0; i < M; i++) mass[i] = m.mass.at(m.type[i]);  // cuda/SELM_Lagrangian_LAMMPS.cu:65-69
  if ((rc = selm_set_particles(s, M, m.x.data(), m.v.data(), mass.data()))) {
    selm_destroy(s);
    return rc;
  }
  selm_topology t{};
  t.natoms = M;
  t.ntypes = m.ntypes;
  t.type = m.type.data();
  t.nbonds = (int)m.bonds.size() / 3;
  t.bond_style = m.bond_style;
  t.nbondtypes = m.nbondtypes;
  t.bonds = m.bonds.data();
  t.bond_coeff = m.bond_coeff.data();
  t.nangles = (int)m.angles.size() / 4;
  t.angle_style = m.angle_style;
  t.nangletypes = m.nangletypes;
  t.angles = m.angles.data();
  t.angle_coeff = m.angle_coeff.data();
  t.pair_style = m.pair_style;
  t.pair_coeff = m.pair_coeff.data();
  for (int q = 0; q < 3; q++) {
    t.special_lj[q] = m.special[q];
    t.body_force[q] = m.body[q];
  }
  if (M > 0 && (rc = selm_set_topology(s, &t))) {
    selm_destroy(s);
    return rc;
  }
  s->case_nsteps = nsteps;
  s->dump_every = m.dump_every;
  s->dump_file = m.dump_file.empty() ? std::string() : (m.dump_file[0] == '/' ? m.dump_file : dir + "/" + m.dump_file);
  *out = s;
  return SELM_OK;
}
