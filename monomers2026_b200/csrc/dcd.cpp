// dcd.cpp - trajectory output in the DCD format LAMMPS' "dump ... dcd" writes.
//
// The reference's cases dump monomer positions through LAMMPS
// (Model.LAMMPS_script: "dump 1 all dcd N file"); its recorded trajectory
// (data/cases/SELM/DIffusion Coefficient/1base.dcd) fixes the layout, which
// this writer follows: Fortran-style records (each framed by its byte length)
//   header  84 B: "CORD", frames, first step, interval, last step, five 0,
//                 timestep (float32), unit-cell flag 1, eight 0, version 24
//   title   2 lines of 80 characters
//   natoms  int32
//   frame   unit cell (6 float64: A, 0, B, 0, 0, C for an orthogonal box),
//           then X, Y, Z as float32 arrays
// The frame count and the last step in the header are rewritten after every
// frame, so the file is complete whenever it is read.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "../../include/selm_b200.h"
#include "selm_engine.h"

struct selm_dcd {
  FILE* f = nullptr;
  int natoms = 0, frames = 0, first = 0, interval = 1;
  double box[3] = {0, 0, 0};
  std::vector<float> buf;
  std::vector<double> host;
};

static void put_i32(FILE* f, int32_t v) { fwrite(&v, 4, 1, f); }

static void put_record(FILE* f, const void* data, int32_t n) {
  put_i32(f, n);
  fwrite(data, 1, (size_t)n, f);
  put_i32(f, n);
}

static void write_header(selm_dcd* d, float dt) {
  unsigned char h[84];
  std::memset(h, 0, sizeof h);
  std::memcpy(h, "CORD", 4);
  int32_t ic[20] = {0};
  ic[0] = d->frames;
  ic[1] = d->first;
  ic[2] = d->interval;
  ic[3] = d->first + (d->frames > 0 ? d->frames - 1 : 0) * d->interval;
  std::memcpy(&ic[9], &dt, 4);  // the timestep, stored as a float32
  ic[10] = 1;                    // a unit cell precedes every frame
  ic[19] = 24;                   // CHARMM format version
  std::memcpy(h + 4, ic, 80);
  put_record(d->f, h, 84);
}

extern "C" int selm_dcd_open(const char* path, int natoms, double dt, int first_step, int interval,
                             const double box_len[3], selm_dcd** out) {
  if (!path || !out || natoms < 0 || interval < 1 || !box_len)
    return selm_fail(SELM_ERR_INVALID, "selm_dcd_open: bad argument");
  *out = nullptr;
  FILE* f = fopen(path, "wb");
  if (!f) return selm_fail(SELM_ERR_IO, std::string("selm_dcd_open: cannot write ") + path);
  selm_dcd* d = new selm_dcd();
  d->f = f;
  d->natoms = natoms;
  d->first = first_step;
  d->interval = interval;
  for (int a = 0; a < 3; a++) d->box[a] = box_len[a];
  write_header(d, (float)dt);
  char title[2][80];
  std::memset(title[0], 0, 80);
  std::snprintf(title[0], 80, "Written by libselm_b200");
  char when[64] = "";
  const std::time_t now = std::time(nullptr);
  std::strftime(when, sizeof when, "%d %B,%Y at %H:%M", std::localtime(&now));
  std::string r = std::string("REMARKS Created ") + when;
  r.resize(80, ' ');
  std::memcpy(title[1], r.data(), 80);
  std::vector<unsigned char> t(4 + 160);
  const int32_t nt = 2;
  std::memcpy(t.data(), &nt, 4);
  std::memcpy(t.data() + 4, title, 160);
  put_record(f, t.data(), (int32_t)t.size());
  const int32_t na = natoms;
  put_record(f, &na, 4);
  d->buf.resize((size_t)natoms);
  fflush(f);
  *out = d;
  return SELM_OK;
}

extern "C" int selm_dcd_open_sim(const char* path, selm_sim* s, int interval, selm_dcd** out) {
  if (!s) return selm_fail(SELM_ERR_INVALID, "sim is NULL");
  const double L = s->hi - s->lo;
  const double box[3] = {L, L, L};
  return selm_dcd_open(path, s->M, s->prm.dt, (int)s->step, interval, box, out);
}

extern "C" int selm_dcd_write(selm_dcd* d, const double* x) {
  if (!d || (!x && d->natoms > 0)) return selm_fail(SELM_ERR_INVALID, "selm_dcd_write: bad argument");
  FILE* f = d->f;
  const double cell[6] = {d->box[0], 0.0, d->box[1], 0.0, 0.0, d->box[2]};
  put_record(f, cell, 48);
  for (int a = 0; a < 3; a++) {
    for (int i = 0; i < d->natoms; i++) d->buf[i] = (float)x[3L * i + a];
    put_record(f, d->buf.data(), (int32_t)(4 * d->natoms));
  }
  d->frames += 1;
  // frame count and last step in the header
  const long end = ftell(f);
  fseek(f, 4 + 4, SEEK_SET);
  const int32_t nset = d->frames, nstep = d->first + (d->frames - 1) * d->interval;
  fwrite(&nset, 4, 1, f);
  fseek(f, 4 + 4 + 12, SEEK_SET);
  fwrite(&nstep, 4, 1, f);
  fseek(f, end, SEEK_SET);
  if (fflush(f) != 0) return selm_fail(SELM_ERR_IO, "selm_dcd_write: write failed");
  return SELM_OK;
}

extern "C" int selm_dcd_write_sim(selm_dcd* d, selm_sim* s) {
  if (!d || !s) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  if (s->M != d->natoms) return selm_fail(SELM_ERR_INVALID, "selm_dcd_write_sim: monomer count differs from the file's");
  d->host.resize(3 * (size_t)d->natoms);
  const int rc = selm_get_particles(s, d->host.data(), nullptr, nullptr);
  if (rc) return rc;
  return selm_dcd_write(d, d->host.data());
}

extern "C" int selm_dcd_close(selm_dcd* d) {
  if (!d) return SELM_OK;
  const int bad = d->f ? fclose(d->f) : 0;
  delete d;
  return bad ? selm_fail(SELM_ERR_IO, "selm_dcd_close: close failed") : SELM_OK;
}

extern "C" int selm_case_dump(selm_sim* s, int* every, char* file, int len) {
  if (!s || !every) return selm_fail(SELM_ERR_INVALID, "NULL argument");
  *every = s->dump_every;
  if (file && len > 0) {
    std::strncpy(file, s->dump_file.c_str(), (size_t)len - 1);
    file[len - 1] = '\0';
  }
  return SELM_OK;
}
