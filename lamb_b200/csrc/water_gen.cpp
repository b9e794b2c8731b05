// Synthetic water-box matrices in LAMB's single-rank sector layout.
// Declarations and the layout contract are in include/lamb_gen.h.
#include "lamb_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(const std::string& m) {
  g_err = m;
  return 1;
}

// splitmix64: seeding and the counter-based value hash.
inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// xoshiro256** stream for the geometry.
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t z = seed;
    for (auto& w : s) { z += 0x9e3779b97f4a7c15ull; w = mix64(z); }
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0,1)
};

// Uniform [-1,1) from (seed, i, j, p, q): a hash chain, independent of
// generation order so that any subset of blocks can be regenerated.
inline double hash_u11(uint64_t seed, uint64_t i, uint64_t j, uint32_t p, uint32_t q) {
  uint64_t h = mix64(seed ^ 0x5851f42d4c957f2dull);
  h = mix64(h ^ i);
  h = mix64(h ^ (j * 0x2545f4914f6cdd1dull));
  h = mix64(h ^ (((uint64_t)p << 32) | q));
  return (double)(h >> 11) * 0x1.0p-52 - 1.0;
}

inline double min_image(double d, double L) { return d - L * std::nearbyint(d / L); }

}  // namespace

struct lamb_gen_geom {
  int32_t n_mol = 0, n_atoms = 0, n_sub = 2;
  double box = 0, cutoff = 0;
  std::vector<double> pos;        // 3*n_atoms
  std::vector<int8_t> blk;        // n_atoms
  std::vector<int32_t> subset;    // 1-based
  std::vector<int32_t> local;     // 0-based local index within the subset
  std::vector<int32_t> sub_count; // atoms per subset
  std::vector<std::vector<int32_t>> sub_atoms;  // global atom ids per subset, in global order
  // Neighbour lists (sorted by j), including i itself.
  std::vector<int64_t> nb_p;      // n_atoms+1
  std::vector<int32_t> nb_j;
  std::vector<double> nb_r;
};

struct lamb_gen_matrix {
  const lamb_gen_geom* geom = nullptr;
  struct Sector {
    int32_t sr, sc, nr, nc;
    std::vector<int8_t> rbs, cbs;
    std::vector<int64_t> row_p;
    std::vector<int16_t> col_i;
    std::vector<int64_t> extents;
    std::vector<double> data;
  };
  std::vector<Sector> sectors;
};

extern "C" {

const char* lamb_gen_last_error(void) { return g_err.c_str(); }

int32_t lamb_gen_water_geometry(int32_t n_mol, double box, double cutoff, int32_t blk_o, int32_t blk_h,
                                uint64_t seed, double min_oo, int32_t n_x_cubes, lamb_gen_geom** out) {
  if (!out) return fail("null output");
  *out = nullptr;
  if (n_mol <= 0 || box <= 0 || cutoff <= 0 || blk_o < 0 || blk_o > 127 || blk_h < 0 || blk_h > 127 ||
      n_x_cubes < 1 || min_oo < 0)
    return fail("invalid water-box parameters");
  auto* g = new lamb_gen_geom;
  g->n_mol = n_mol;
  g->n_atoms = 3 * n_mol;
  g->box = box;
  g->cutoff = cutoff;
  g->n_sub = n_x_cubes;
  const double L = box;
  Rng rng(seed);
  // Random sequential insertion of oxygens on a cell grid (cell >= min_oo).
  int nc = std::max(1, (int)std::floor(L / std::max(min_oo, 1e-9)));
  nc = std::min(nc, 256);
  const double cell = L / nc;
  std::vector<std::vector<int32_t>> cells((size_t)nc * nc * nc);
  std::vector<double> O(3 * (size_t)n_mol);
  auto cell_of = [&](double x) { int c = (int)(x / cell); return std::min(std::max(c, 0), nc - 1); };
  const double min2 = min_oo * min_oo;
  const int reach = (int)std::ceil(min_oo / cell);
  for (int m = 0; m < n_mol; ++m) {
    bool placed = false;
    for (int attempt = 0; attempt < 2000000 && !placed; ++attempt) {
      double x[3] = {rng.uniform() * L, rng.uniform() * L, rng.uniform() * L};
      int c[3] = {cell_of(x[0]), cell_of(x[1]), cell_of(x[2])};
      bool ok = true;
      if (nc <= 2 * reach + 1) {
        for (int o = 0; o < m && ok; ++o) {
          double d2 = 0;
          for (int a = 0; a < 3; ++a) { double d = min_image(x[a] - O[3 * o + a], L); d2 += d * d; }
          ok = d2 >= min2;
        }
      } else {
        for (int dx = -reach; dx <= reach && ok; ++dx)
          for (int dy = -reach; dy <= reach && ok; ++dy)
            for (int dz = -reach; dz <= reach && ok; ++dz) {
              int cx = (c[0] + dx + nc) % nc, cy = (c[1] + dy + nc) % nc, cz = (c[2] + dz + nc) % nc;
              for (int o : cells[((size_t)cx * nc + cy) * nc + cz]) {
                double d2 = 0;
                for (int a = 0; a < 3; ++a) { double d = min_image(x[a] - O[3 * o + a], L); d2 += d * d; }
                if (d2 < min2) { ok = false; break; }
              }
            }
      }
      if (ok) {
        for (int a = 0; a < 3; ++a) O[3 * m + a] = x[a];
        cells[((size_t)c[0] * nc + c[1]) * nc + c[2]].push_back(m);
        placed = true;
      }
    }
    if (!placed) { delete g; return fail("could not place molecule (box too dense)"); }
  }
  // Orientation: uniform random rotation (Shoemake quaternion).
  const double r_oh = 0.96, half = 0.5 * 104.5 * M_PI / 180.0;
  const double h1[3] = {r_oh * std::sin(half), r_oh * std::cos(half), 0.0};
  const double h2[3] = {-r_oh * std::sin(half), r_oh * std::cos(half), 0.0};
  g->pos.resize(3 * (size_t)g->n_atoms);
  g->blk.resize(g->n_atoms);
  for (int m = 0; m < n_mol; ++m) {
    double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
    double qa = std::sqrt(1 - u1) * std::sin(2 * M_PI * u2), qb = std::sqrt(1 - u1) * std::cos(2 * M_PI * u2);
    double qc = std::sqrt(u1) * std::sin(2 * M_PI * u3), qd = std::sqrt(u1) * std::cos(2 * M_PI * u3);
    // rotation matrix of unit quaternion (w=qd, x=qa, y=qb, z=qc)
    double w = qd, X = qa, Y = qb, Z = qc;
    double R[3][3] = {{1 - 2 * (Y * Y + Z * Z), 2 * (X * Y - Z * w), 2 * (X * Z + Y * w)},
                      {2 * (X * Y + Z * w), 1 - 2 * (X * X + Z * Z), 2 * (Y * Z - X * w)},
                      {2 * (X * Z - Y * w), 2 * (Y * Z + X * w), 1 - 2 * (X * X + Y * Y)}};
    const double* hs[2] = {h1, h2};
    for (int a = 0; a < 3; ++a) g->pos[3 * (3 * m) + a] = O[3 * m + a];
    for (int h = 0; h < 2; ++h)
      for (int a = 0; a < 3; ++a) {
        double v = O[3 * m + a] + R[a][0] * hs[h][0] + R[a][1] * hs[h][1] + R[a][2] * hs[h][2];
        v = v - L * std::floor(v / L);
        if (v >= L) v -= L;
        g->pos[3 * (3 * m + 1 + h) + a] = v;
      }
    g->blk[3 * m] = (int8_t)blk_o;
    g->blk[3 * m + 1] = (int8_t)blk_h;
    g->blk[3 * m + 2] = (int8_t)blk_h;
  }
  // Subsets: float32 rule of lamb_partition_which_cube1 with n_x_cubes cubes along x.
  g->subset.resize(g->n_atoms);
  g->local.resize(g->n_atoms);
  g->sub_count.assign(n_x_cubes, 0);
  g->sub_atoms.assign(n_x_cubes, {});
  const float mult = (float)n_x_cubes / (float)L;
  for (int i = 0; i < g->n_atoms; ++i) {
    float x = (float)g->pos[3 * i];
    int c = (int)(x * mult);  // Fortran int(): truncation toward zero
    c = c % n_x_cubes;
    if (c < 0) c += n_x_cubes;
    g->subset[i] = c + 1;
    g->local[i] = g->sub_count[c]++;
    g->sub_atoms[c].push_back(i);
  }
  for (int s = 0; s < n_x_cubes; ++s)
    if (g->sub_count[s] > 32767) { delete g; return fail("subset exceeds the int16 local-atom range"); }
  // Neighbour lists with one minimum image per pair.
  const int na = g->n_atoms;
  const double rc2 = cutoff * cutoff;
  std::vector<std::vector<std::pair<int32_t, double>>> nb(na);
  int ncn = std::max(1, (int)std::floor(L / cutoff));
  ncn = std::min(ncn, 128);
  if (ncn < 3) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < na; ++j) {
        double d2 = 0;
        for (int a = 0; a < 3; ++a) { double d = min_image(g->pos[3 * i + a] - g->pos[3 * j + a], L); d2 += d * d; }
        if (d2 < rc2) nb[i].push_back({j, std::sqrt(d2)});
      }
  } else {
    const double cl = L / ncn;
    std::vector<std::vector<int32_t>> cl_atoms((size_t)ncn * ncn * ncn);
    auto cc = [&](double x) { int c = (int)(x / cl); return std::min(std::max(c, 0), ncn - 1); };
    for (int i = 0; i < na; ++i)
      cl_atoms[((size_t)cc(g->pos[3 * i]) * ncn + cc(g->pos[3 * i + 1])) * ncn + cc(g->pos[3 * i + 2])].push_back(i);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < na; ++i) {
      int c0 = cc(g->pos[3 * i]), c1 = cc(g->pos[3 * i + 1]), c2 = cc(g->pos[3 * i + 2]);
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            int x = (c0 + dx + ncn) % ncn, y = (c1 + dy + ncn) % ncn, z = (c2 + dz + ncn) % ncn;
            for (int j : cl_atoms[((size_t)x * ncn + y) * ncn + z]) {
              double d2 = 0;
              for (int a = 0; a < 3; ++a) { double d = min_image(g->pos[3 * i + a] - g->pos[3 * j + a], L); d2 += d * d; }
              if (d2 < rc2) nb[i].push_back({j, std::sqrt(d2)});
            }
          }
      std::sort(nb[i].begin(), nb[i].end());
    }
  }
  g->nb_p.resize(na + 1);
  g->nb_p[0] = 0;
  for (int i = 0; i < na; ++i) g->nb_p[i + 1] = g->nb_p[i] + (int64_t)nb[i].size();
  g->nb_j.resize(g->nb_p[na]);
  g->nb_r.resize(g->nb_p[na]);
  for (int i = 0; i < na; ++i) {
    std::sort(nb[i].begin(), nb[i].end());
    for (size_t t = 0; t < nb[i].size(); ++t) {
      g->nb_j[g->nb_p[i] + t] = nb[i][t].first;
      g->nb_r[g->nb_p[i] + t] = nb[i][t].second;
    }
  }
  *out = g;
  return 0;
}

int32_t lamb_gen_geom_free(lamb_gen_geom* geom) {
  delete geom;
  return 0;
}

int32_t lamb_gen_geom_n_atoms(const lamb_gen_geom* g) { return g ? g->n_atoms : -1; }
int64_t lamb_gen_geom_n_pairs(const lamb_gen_geom* g) { return g ? g->nb_p.back() : -1; }

int32_t lamb_gen_geom_atoms(const lamb_gen_geom* g, double* positions, int8_t* blk, int32_t* subset, int32_t* local) {
  if (!g) return fail("null geometry");
  if (positions) std::memcpy(positions, g->pos.data(), sizeof(double) * g->pos.size());
  if (blk) std::memcpy(blk, g->blk.data(), g->blk.size());
  if (subset) std::memcpy(subset, g->subset.data(), sizeof(int32_t) * g->subset.size());
  if (local) std::memcpy(local, g->local.data(), sizeof(int32_t) * g->local.size());
  return 0;
}

int32_t lamb_gen_water_matrix(const lamb_gen_geom* g, uint64_t seed, double decay, int32_t symmetric,
                              lamb_gen_matrix** out) {
  if (!g || !out) return fail("null argument");
  if (!(decay > 0)) return fail("decay must be positive");
  auto* M = new lamb_gen_matrix;
  M->geom = g;
  const int S = g->n_sub;
  M->sectors.resize((size_t)S * S);
  for (int m = 0; m < S; ++m)
    for (int n = 0; n < S; ++n) {
      auto& sec = M->sectors[(size_t)m * S + n];
      sec.sr = m + 1;
      sec.sc = n + 1;
      sec.nr = g->sub_count[m];
      sec.nc = g->sub_count[n];
      sec.rbs.resize(sec.nr);
      sec.cbs.resize(sec.nc);
      for (int r = 0; r < sec.nr; ++r) sec.rbs[r] = g->blk[g->sub_atoms[m][r]];
      for (int c = 0; c < sec.nc; ++c) sec.cbs[c] = g->blk[g->sub_atoms[n][c]];
      sec.row_p.assign(sec.nr + 1, 0);
      // Count blocks per local row (neighbours of the row atom that fall in subset n).
      for (int r = 0; r < sec.nr; ++r) {
        int i = g->sub_atoms[m][r];
        int64_t cnt = 0;
        for (int64_t t = g->nb_p[i]; t < g->nb_p[i + 1]; ++t) cnt += (g->subset[g->nb_j[t]] == n + 1);
        sec.row_p[r + 1] = sec.row_p[r] + cnt;
      }
      const int64_t nb = sec.row_p[sec.nr];
      sec.col_i.resize(nb);
      sec.extents.resize(2 * nb);
      // Column order within a row: ascending local column.  Neighbour lists are
      // sorted by global id, and local ids within a subset follow global order.
      std::vector<int64_t> doff(sec.nr + 1, 0);
      for (int r = 0; r < sec.nr; ++r) {
        int i = g->sub_atoms[m][r];
        int64_t sz = 0;
        for (int64_t t = g->nb_p[i]; t < g->nb_p[i + 1]; ++t)
          if (g->subset[g->nb_j[t]] == n + 1) sz += (int64_t)g->blk[i] * g->blk[g->nb_j[t]];
        doff[r + 1] = doff[r] + sz;
      }
      sec.data.resize(doff[sec.nr]);
#pragma omp parallel for schedule(dynamic, 8)
      for (int r = 0; r < sec.nr; ++r) {
        const int i = g->sub_atoms[m][r];
        const int bi = g->blk[i];
        int64_t b = sec.row_p[r];
        int64_t off = doff[r];
        for (int64_t t = g->nb_p[i]; t < g->nb_p[i + 1]; ++t) {
          const int j = g->nb_j[t];
          if (g->subset[j] != n + 1) continue;
          const int bj = g->blk[j];
          sec.col_i[b] = (int16_t)(g->local[j] + 1);
          sec.extents[2 * b] = off + 1;
          sec.extents[2 * b + 1] = off + (int64_t)bi * bj;
          const double f = std::exp(-g->nb_r[t] / decay);
          double* d = sec.data.data() + off;
          for (int q = 0; q < bj; ++q)
            for (int p = 0; p < bi; ++p) {
              double v;
              if (i == j) {
                v = 0.5 * (hash_u11(seed, i, i, p, q) + hash_u11(seed, i, i, q, p)) + (p == q ? 1.0 : 0.0);
              } else if (symmetric && i > j) {
                v = hash_u11(seed, j, i, q, p) * f;
              } else {
                v = hash_u11(seed, i, j, p, q) * f;
              }
              d[(size_t)q * bi + p] = v;  // column-major block
            }
          off += (int64_t)bi * bj;
          ++b;
        }
      }
    }
  *out = M;
  return 0;
}

int32_t lamb_gen_matrix_free(lamb_gen_matrix* m) {
  delete m;
  return 0;
}

int32_t lamb_gen_matrix_n_sectors(const lamb_gen_matrix* m) { return m ? (int32_t)m->sectors.size() : -1; }

int32_t lamb_gen_matrix_sector(const lamb_gen_matrix* m, int32_t s, lamb_c_sector* o) {
  if (!m || !o || s < 0 || s >= (int32_t)m->sectors.size()) return fail("bad sector query");
  const auto& sec = m->sectors[s];
  o->subset_row = sec.sr;
  o->subset_col = sec.sc;
  o->n_rows = sec.nr;
  o->n_cols = sec.nc;
  o->row_blk_sizes = sec.rbs.data();
  o->col_blk_sizes = sec.cbs.data();
  o->row_p = sec.row_p.data();
  o->col_i = sec.col_i.data();
  o->extents = sec.extents.data();
  o->data = sec.data.data();
  o->n_blks = (int64_t)sec.col_i.size();
  o->data_len = (int64_t)sec.data.size();
  return 0;
}

}  // extern "C"
