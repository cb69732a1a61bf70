// Grids on disk: a binary cache so that a restart reuses grids instead of rebuilding them, and the reference's cube
// writer for viewers.
//
// The reference rebuilds every interpolation grid when a run starts or restarts: grids are not part of its archive
// (system.cpp:1558-1562 sizes empty slots and createInterpolationGrids refills them). rg_grid_save / rg_grid_load store
// one grid with a 64-bit fingerprint of every input that determines it (rg_grid_fingerprint), a shape check and a
// checksum of the values, so that a stale or damaged file is a cache miss (RG_ERR_CACHE_MISS), never wrong data.
// rg_grid_write_cube writes the energy channel in the format of InterpolationEnergyGrid::writeOutput
// (interpolation_energy_grid.cpp:4760-4789). Host code only: none of these calls touches the device.
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace
{
// FNV-1a, 64 bit
struct Fnv
{
  uint64_t h = 1469598103934665603ull;
  void bytes(const void* p, size_t n)
  {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i)
    {
      h ^= c[i];
      h *= 1099511628211ull;
    }
  }
  template <typename T>
  void value(const T& v)
  {
    bytes(&v, sizeof(T));
  }
};

constexpr char kMagic[8] = {'R', 'G', 'G', 'R', 'I', 'D', '\0', '\1'};
constexpr uint32_t kVersion = 1;

struct FileHeader
{
  char magic[8];
  uint32_t version;
  int32_t scheme;
  int32_t nx, ny, nz;
  int32_t pad;
  uint64_t fingerprint;
  uint64_t values;    // doubles that follow
  uint64_t checksum;  // FNV-1a of the values' bytes
  double cell[9];
};
static_assert(sizeof(FileHeader) == 8 + 4 + 4 + 12 + 4 + 24 + 72, "packed header");

bool validScheme(int s) { return s == RG_SCHEME_TRICUBIC || s == RG_SCHEME_TRIQUINTIC; }

// EnergyToKelvin (units.cpp:91-98): the internal energy unit (10 J/mol) in K
double energyToKelvin() { return rg::energyConversionFactor() * 6.0221419947e23 / 8.314464919; }

// shortest round-trip decimal form of a double, as std::format's "{}" writes it
void appendDouble(std::string& out, double v)
{
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof(buf), v);
  out.append(buf, r.ptr);
}
}  // namespace

extern "C"
{
uint64_t rg_grid_fingerprint(int grid_type, int scheme, int flags, const rg_forcefield* ff, const rg_box* unit_cell,
                             const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, int nx, int ny, int nz)
{
  Fnv f;
  f.value(kVersion);
  f.value(grid_type);
  f.value(scheme);
  f.value(flags);
  f.value(nx);
  f.value(ny);
  f.value(nz);
  if (unit_cell)
  {
    f.bytes(unit_cell->cell, sizeof(unit_cell->cell));
    f.value(unit_cell->triclinic);
  }
  if (ff)
  {
    f.value(ff->cutoff_framework_vdw);
    f.value(ff->ewald_alpha);
    f.value(ff->overlap_criteria);
    f.value(ff->n_types);
    // the probe's row of the mixed pair table (Lennard-Jones grids); the Ewald grid does not depend on it
    if (grid_type != RG_GRID_EWALD_REAL && probe_type >= 0 && probe_type < ff->n_types && ff->epsilon && ff->sigma &&
        ff->shift)
    {
      f.value(probe_type);
      for (int t = 0; t < ff->n_types; ++t)
      {
        const int idx = probe_type * ff->n_types + t;
        f.value(ff->epsilon[idx]);
        f.value(ff->sigma[idx]);
        f.value(ff->shift[idx]);
      }
    }
  }
  f.value(n_unit_atoms);
  for (int a = 0; a < n_unit_atoms && unit_atoms; ++a)
  {
    const rg_atom& at = unit_atoms[a];
    f.value(at.x);
    f.value(at.y);
    f.value(at.z);
    f.value(at.charge);
    f.value(at.type);
  }
  return f.h;
}

rg_status rg_grid_save(const char* path, uint64_t fingerprint, int scheme, const rg_box* unit_cell, int nx, int ny,
                       int nz, const double* data)
{
  if (!path || !unit_cell || !data || !validScheme(scheme) || nx < 2 || ny < 2 || nz < 2)
    return RG_ERR_INVALID_ARGUMENT;
  FileHeader h{};
  std::memcpy(h.magic, kMagic, sizeof(kMagic));
  h.version = kVersion;
  h.scheme = scheme;
  h.nx = nx;
  h.ny = ny;
  h.nz = nz;
  h.fingerprint = fingerprint;
  h.values = static_cast<uint64_t>(scheme) * nx * ny * nz;
  Fnv sum;
  sum.bytes(data, sizeof(double) * h.values);
  h.checksum = sum.h;
  std::memcpy(h.cell, unit_cell->cell, sizeof(h.cell));
  // write to a temporary name, then rename: a reader never sees a half-written file
  const std::string tmp = std::string(path) + ".tmp";
  FILE* fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) return RG_ERR_IO;
  bool ok = std::fwrite(&h, sizeof(h), 1, fp) == 1 &&
            std::fwrite(data, sizeof(double), h.values, fp) == h.values;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path) != 0)
  {
    std::remove(tmp.c_str());
    return RG_ERR_IO;
  }
  return RG_OK;
}

rg_status rg_grid_load(const char* path, uint64_t fingerprint, int scheme, int nx, int ny, int nz, double* data)
{
  if (!path || !data || !validScheme(scheme) || nx < 2 || ny < 2 || nz < 2) return RG_ERR_INVALID_ARGUMENT;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return RG_ERR_CACHE_MISS;
  FileHeader h{};
  rg_status st = RG_OK;
  const uint64_t want = static_cast<uint64_t>(scheme) * nx * ny * nz;
  if (std::fread(&h, sizeof(h), 1, fp) != 1 || std::memcmp(h.magic, kMagic, sizeof(kMagic)) != 0 ||
      h.version != kVersion || h.scheme != scheme || h.nx != nx || h.ny != ny || h.nz != nz ||
      h.fingerprint != fingerprint || h.values != want)
    st = RG_ERR_CACHE_MISS;
  if (!st && std::fread(data, sizeof(double), want, fp) != want) st = RG_ERR_CACHE_MISS;
  std::fclose(fp);
  if (!st)
  {
    Fnv sum;
    sum.bytes(data, sizeof(double) * want);
    if (sum.h != h.checksum) st = RG_ERR_CACHE_MISS;
  }
  return st;
}

rg_status rg_grid_write_cube(const char* path, int scheme, const double* data, int nx, int ny, int nz,
                             const rg_box* unit_cell, const double* origin)
{
  if (!path || !data || !unit_cell || !validScheme(scheme) || nx < 2 || ny < 2 || nz < 2)
    return RG_ERR_INVALID_ARGUMENT;
  FILE* fp = std::fopen(path, "w");
  if (!fp) return RG_ERR_IO;
  const double o[3] = {origin ? origin[0] : 0.0, origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
  const int n[3] = {nx, ny, nz};
  std::string out = "Cube interpolation file\nWritten by RASPA-3\n1 ";
  for (int d = 0; d < 3; ++d)
  {
    appendDouble(out, o[d]);
    out += d < 2 ? " " : "\n";
  }
  // one line per cell vector: the negative point count (Angstrom units) and the vector over the point count
  for (int c = 0; c < 3; ++c)
  {
    out += std::to_string(-n[c]);
    for (int r = 0; r < 3; ++r)
    {
      out += ' ';
      appendDouble(out, unit_cell->cell[3 * c + r] / static_cast<double>(n[c]));
    }
    out += '\n';
  }
  out += "1 0.0 0.0 0.0 0.0\n";
  const double k = energyToKelvin();
  const size_t npts = static_cast<size_t>(nx) * ny * nz;
  bool ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
  out.clear();
  for (size_t p = 0; p < npts && ok; ++p)
  {
    appendDouble(out, data[static_cast<size_t>(scheme) * p] * k);
    out += '\n';
    if (out.size() > (1u << 20) || p + 1 == npts)
    {
      ok = std::fwrite(out.data(), 1, out.size(), fp) == out.size();
      out.clear();
    }
  }
  ok = (std::fclose(fp) == 0) && ok;
  return ok ? RG_OK : RG_ERR_IO;
}
}
