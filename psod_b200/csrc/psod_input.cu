// psod_input.cu -- the reference's binary particle reader (host code only).
//
// Built without HDF5, the reference's SOD driver reads each zone's particles
// from the cube files of the FoF step, "<root>_cube_NNNNN" (main:455-534):
// Fortran unformatted sequential files whose records are nloc, the writer's
// rank, the cube bounds, the positions, the velocities and the IDs.  For a
// zone it opens the 27 cubes around it (periodic) and keeps the particles
// inside the zone plus its buffer.  psod_read_cube_zone restates that: the
// same file list and order, the same FP64 distance test, particles kept in
// file order, so that the arrays it fills are the reference's posf / velf /
// idf and can go straight to psod_load_particles.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "psod_internal.cuh"

namespace {

// One Fortran unformatted sequential record.  gfortran writes a record of
// 2^31 bytes or more as subrecords whose leading marker is negative while
// more subrecords follow; the payloads are concatenated.
bool read_record(FILE *f, std::vector<unsigned char> &out) {
  out.clear();
  while (true) {
    int32_t head = 0, tail = 0;
    if (std::fread(&head, 4, 1, f) != 1) return false;
    const bool more = head < 0;
    const size_t len = (size_t)(more ? -(int64_t)head : (int64_t)head);
    const size_t at = out.size();
    out.resize(at + len);
    if (len && std::fread(out.data() + at, 1, len, f) != len) return false;
    if (std::fread(&tail, 4, 1, f) != 1) return false;
    if (!more) return true;
  }
}

struct CubeFile {
  int32_t nloc = 0;
  std::vector<float> pos, vel;
  std::vector<int64_t> id;
};

// the records of one cube file; with positions only when want_all is false
// (the reference's counting pass reads no further, main:463-468)
int read_cube(const std::string &path, int id_bytes, bool want_all, CubeFile &c) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return PSOD_ERR_IO;
  std::vector<unsigned char> r;
  int st = PSOD_ERR_IO;
  do {
    if (!read_record(f, r) || r.size() != 4) break;  // nloc
    std::memcpy(&c.nloc, r.data(), 4);
    if (c.nloc < 0) break;
    const size_t n = (size_t)c.nloc;
    if (!read_record(f, r) || r.size() != 4) break;   // proc_ID
    if (!read_record(f, r) || r.size() != 24) break;  // mintmp/maxtmp, 3 x 2 real(4)
    if (!read_record(f, r) || r.size() != 12 * n) break;
    c.pos.resize(3 * n);
    if (n) std::memcpy(c.pos.data(), r.data(), 12 * n);
    if (want_all) {
      if (!read_record(f, r) || r.size() != 12 * n) break;
      c.vel.resize(3 * n);
      if (n) std::memcpy(c.vel.data(), r.data(), 12 * n);
      if (!read_record(f, r) || r.size() != (size_t)id_bytes * n) break;
      c.id.resize(n);
      for (size_t i = 0; i < n; i++) {
        if (id_bytes == 8) {
          std::memcpy(&c.id[i], r.data() + 8 * i, 8);
        } else {
          int32_t v;
          std::memcpy(&v, r.data() + 4 * i, 4);
          c.id[i] = v;
        }
      }
    }
    st = PSOD_OK;
  } while (false);
  std::fclose(f);
  return st;
}

struct ZoneSelect {
  double xc[3], rsmall[3], rlarge[3];
  // the reference's test (main:471-479): on every axis the distance to the
  // zone centre is below rsmall or (periodic image) above rlarge
  bool keep(const float *p) const {
    for (int a = 0; a < 3; a++) {
      const double d = std::fabs((double)p[a] - xc[a]);
      if (!(d < rsmall[a] || d > rlarge[a])) return false;
    }
    return true;
  }
};

}  // namespace

extern "C" int psod_read_cube_zone(const char *root, int32_t ncpu, int32_t nzone, int32_t nx, int32_t nxbuffer,
                                   int32_t id_bytes, int64_t capacity, int64_t *npart, float *pos, float *vel,
                                   int64_t *id) {
  if (!root || !npart || ncpu < 1 || nzone < 0 || nzone >= ncpu || nx < 1 || nxbuffer < 0 ||
      (id_bytes != 4 && id_bytes != 8))
    return PSOD_ERR_ARG;
  // cubes per side and the zone's 3-D index (main:340-347)
  const int nxcpu = (int)std::lround(std::pow((double)ncpu, 1.0 / 3.0));
  if (nxcpu < 1 || (int64_t)nxcpu * nxcpu * nxcpu != ncpu) return PSOD_ERR_ARG;
  const int nycpu = nxcpu, nzcpu = nxcpu;
  const int ix = (int)((double)nzone / (double)(nycpu * nzcpu));
  const int iy = (int)((double)(nzone - ix * nycpu * nzcpu) / (double)nzcpu);
  const int iz = nzone - ix * nycpu * nzcpu - iy * nzcpu;
  const int nxzone = nx / nxcpu;  // main:350
  if (nxzone < 1) return PSOD_ERR_ARG;
  const int nxb = nxbuffer == 0 ? nxzone / 2 : nxbuffer;  // main:380-381
  if (nxb > nxzone) return PSOD_ERR_ARG;                  // main:392-397
  // the 27 cubes around the zone, x outer and z inner (main:363-375); with
  // fewer than three cubes a side the reference lists some twice and loads
  // their particles twice: each distinct cube is read once here
  std::vector<int> files;
  for (int i = ix - 1; i <= ix + 1; i++)
    for (int j = iy - 1; j <= iy + 1; j++)
      for (int k = iz - 1; k <= iz + 1; k++) {
        const int it = i < 0 ? nxcpu - 1 : i, jt = j < 0 ? nycpu - 1 : j, kt = k < 0 ? nzcpu - 1 : k;
        const int f = (kt % nzcpu) + (jt % nycpu) * nzcpu + (it % nxcpu) * nzcpu * nycpu;
        bool seen = false;
        for (int g : files) seen = seen || g == f;
        if (!seen) files.push_back(f);
      }
  // zone centre and half-widths with buffer (main:421-439)
  ZoneSelect z;
  const int izone[3] = {ix, iy, iz};
  for (int a = 0; a < 3; a++) {
    const double lo = (double)izone[a] / (double)nxcpu, hi = (double)(izone[a] + 1) / (double)nxcpu;
    z.xc[a] = (lo + hi) / 2.0;
    z.rsmall[a] = (0.5 + (double)nxb / (double)nxzone) / (double)nxcpu;
    z.rlarge[a] = 1.0 - z.rsmall[a];
  }
  const bool fill = pos != nullptr;
  if (fill && !id) return PSOD_ERR_ARG;
  int64_t count = 0;
  for (int f : files) {
    char num[16];
    std::snprintf(num, sizeof num, "%05d", f);
    CubeFile c;
    const int st = read_cube(std::string(root) + "_cube_" + num, id_bytes, fill, c);
    if (st) return st;
    for (int32_t i = 0; i < c.nloc; i++) {
      if (!z.keep(&c.pos[3 * (size_t)i])) continue;
      if (fill) {
        if (count >= capacity) return PSOD_ERR_ARG;
        std::memcpy(pos + 3 * count, &c.pos[3 * (size_t)i], 12);
        if (vel) std::memcpy(vel + 3 * count, &c.vel[3 * (size_t)i], 12);
        id[count] = c.id[i];
      }
      count++;
    }
  }
  *npart = count;
  return PSOD_OK;
}

// The driver's particle selection for one zone (main:573-600): the zone's
// particles with their buffer, by the same FP64 test as the cube reader.
extern "C" int psod_select_zone(int32_t nx, int32_t nxcpu, int32_t nzone, int32_t nxbuffer, const float *pos,
                                int64_t n, uint8_t *keep, int64_t *nkeep) {
  if (nx < 1 || nxcpu < 1 || nx % nxcpu != 0 || nzone < 0 || (int64_t)nzone >= (int64_t)nxcpu * nxcpu * nxcpu ||
      nxbuffer < 0 || n < 0 || (n > 0 && (!pos || !keep)) || !nkeep)
    return PSOD_ERR_ARG;
  const int nxzone = nx / nxcpu;                          // main:350
  const int nxb = nxbuffer == 0 ? nxzone / 2 : nxbuffer;  // main:380-381
  if (nxb > nxzone) return PSOD_ERR_ARG;                  // main:392-397
  // zone indices (main:344-346), centre and half-widths with buffer (main:421-439)
  const int izone[3] = {nzone / (nxcpu * nxcpu), (nzone / nxcpu) % nxcpu, nzone % nxcpu};
  ZoneSelect z;
  for (int a = 0; a < 3; a++) {
    const double lo = (double)izone[a] / (double)nxcpu, hi = (double)(izone[a] + 1) / (double)nxcpu;
    z.xc[a] = (lo + hi) / 2.0;
    z.rsmall[a] = (0.5 + (double)nxb / (double)nxzone) / (double)nxcpu;
    z.rlarge[a] = 1.0 - z.rsmall[a];
  }
  int64_t count = 0;
  for (int64_t i = 0; i < n; i++) {
    const bool k = z.keep(pos + 3 * i);
    keep[i] = k ? 1 : 0;
    count += k ? 1 : 0;
  }
  *nkeep = count;
  return PSOD_OK;
}
