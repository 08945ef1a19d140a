// psod_output.cu -- the reference's binary halo outputs (host code only).
//
// spherover writes, when built without HDF5, two Fortran unformatted
// sequential files per zone (main:2230-2259): "masst" (one record per halo:
// ID, N_delta, centre) and "strct" (per halo its N_delta and its members'
// positions, velocities, IDs and optional potential / force in ascending
// distance).  A sequential unformatted record is its payload between two
// copies of its byte length as int32, which is how gfortran writes records
// below 2^31 bytes.  These writers produce those files from the halo table
// of psod_get_halos and the zone's particle arrays; they run on the host and
// need no device.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <utility>
#include <vector>

#include "psod_internal.cuh"

namespace {

struct RecordFile {
  FILE *f = nullptr;
  bool ok = true;
  explicit RecordFile(const char *path) : f(std::fopen(path, "wb")) { ok = f != nullptr; }
  ~RecordFile() {
    if (f) std::fclose(f);
  }
  // one record made of `parts` (pointer, bytes) pieces
  void record(std::initializer_list<std::pair<const void *, size_t>> parts) {
    size_t len = 0;
    for (auto &p : parts) len += p.second;
    if (len >= (size_t)1 << 31) {  // gfortran would split it into subrecords
      ok = false;
      return;
    }
    const int32_t m = (int32_t)len;
    ok = ok && std::fwrite(&m, 4, 1, f) == 1;
    for (auto &p : parts)
      if (p.second) ok = ok && std::fwrite(p.first, 1, p.second, f) == p.second;
    ok = ok && std::fwrite(&m, 4, 1, f) == 1;
  }
  bool close() {
    if (!f) return false;
    const bool good = ok && std::fclose(f) == 0;
    f = nullptr;
    return good;
  }
};

bool table_ok(const psod_halo_table *t, int64_t nhalo) {
  return t && nhalo >= 0 && nhalo < ((int64_t)1 << 31) && (nhalo == 0 || (t->halo_mass && t->member_offset));
}

// Every record is checked before the file is opened, so an invalid table
// leaves no partly written file behind.
bool masses_ok(const psod_halo_table *t, int64_t nhalo) {
  for (int64_t h = 0; h < nhalo; h++)
    if (t->halo_mass[h] < 0 || t->halo_mass[h] > INT32_MAX) return false;
  return true;
}

bool members_ok(const psod_halo_table *t, int64_t nhalo, int64_t n) {
  for (int64_t h = 0; h < nhalo; h++) {
    const int64_t m = t->halo_mass[h], o = t->member_offset[h];
    if (m < 0 || 12 * m >= ((int64_t)1 << 31) || o < 0 || t->member_offset[h + 1] - o != m) return false;
    for (int64_t j = 0; j < m; j++) {
      const int64_t q = t->member_index[o + j];
      if (q < 0 || q >= n) return false;
    }
  }
  return true;
}

}  // namespace

extern "C" {

int psod_write_masst(const char *path, const psod_halo_table *t, int64_t nhalo) {
  if (!path || !table_ok(t, nhalo) || (nhalo > 0 && (!t->halo_id || !t->halo_center))) return PSOD_ERR_ARG;
  if (!masses_ok(t, nhalo)) return PSOD_ERR_ARG;
  RecordFile out(path);
  if (!out.ok) return PSOD_ERR_IO;
  const int32_t namas = (int32_t)nhalo;
  out.record({{&namas, 4}});  // main:2235
  for (int64_t h = 0; h < nhalo; h++) {
    const int64_t id = t->halo_id[h];
    const int32_t mass = (int32_t)t->halo_mass[h];  // masses(i), default integer
    // int(idtab(i),kind=8), masses(i), xctab(i), yctab(i), zctab(i) (main:2237)
    out.record({{&id, 8}, {&mass, 4}, {t->halo_center + 3 * h, 12}});
  }
  return out.close() ? PSOD_OK : PSOD_ERR_IO;
}

int psod_write_strct(const char *path, const psod_halo_table *t, int64_t nhalo, int64_t n, const float *pos,
                     const float *vel, const int64_t *id, const float *pot, const float *force) {
  if (!path || !table_ok(t, nhalo) || n < 0 || (nhalo > 0 && (!t->member_index || !pos || !id)))
    return PSOD_ERR_ARG;
  if (!members_ok(t, nhalo, n)) return PSOD_ERR_ARG;
  RecordFile out(path);
  if (!out.ok) return PSOD_ERR_IO;
  const int32_t namas = (int32_t)nhalo;
  out.record({{&namas, 4}});  // main:2247
  std::vector<float> buf3, buf1;
  std::vector<int64_t> bufi;
  for (int64_t h = 0; h < nhalo; h++) {
    const int64_t m = t->halo_mass[h], o = t->member_offset[h];
    const int32_t mass = (int32_t)m;
    out.record({{&mass, 4}});  // main:2250
    buf3.resize((size_t)(3 * m));
    bufi.resize((size_t)m);
    for (int64_t j = 0; j < m; j++) {
      const int64_t q = t->member_index[o + j];
      std::memcpy(&buf3[3 * j], pos + 3 * q, 12);
      bufi[j] = id[q];
    }
    out.record({{buf3.data(), (size_t)(12 * m)}});  // positions, box units (main:2251)
    for (int64_t j = 0; j < m; j++) {
      const int64_t q = t->member_index[o + j];
      if (vel) std::memcpy(&buf3[3 * j], vel + 3 * q, 12);
      else buf3[3 * j] = buf3[3 * j + 1] = buf3[3 * j + 2] = 0.f;
    }
    out.record({{buf3.data(), (size_t)(12 * m)}});  // velocities (main:2252)
    out.record({{bufi.data(), (size_t)(8 * m)}});   // IDs (main:2253)
    if (pot) {  // main:2254
      buf1.resize((size_t)m);
      for (int64_t j = 0; j < m; j++) buf1[j] = pot[t->member_index[o + j]];
      out.record({{buf1.data(), (size_t)(4 * m)}});
    }
    if (force) {  // main:2255
      for (int64_t j = 0; j < m; j++) std::memcpy(&buf3[3 * j], force + 3 * t->member_index[o + j], 12);
      out.record({{buf3.data(), (size_t)(12 * m)}});
    }
  }
  return out.close() ? PSOD_OK : PSOD_ERR_IO;
}

}  // extern "C"
