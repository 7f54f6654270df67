// mesh_gen.cpp -- seeded synthetic meshes for the mesh-built octrees.
//
// The reference voxelises laser scans (PLY meshes) that are not part of it;
// these generators make meshes of the sizes the benchmark configurations name:
//   * icosphere: the 20-face icosahedron, each subdivision splitting every
//     triangle into four at its edge midpoints (20 * 4^k faces), vertices
//     pushed to radius r + a * fbm(direction) with 3D value noise;
//   * terrain:   an n x n height field over the unit square, y from 2D fBm.
// Value noise: a hash of the integer lattice point gives a value in [-1, 1],
// interpolated with the smoothstep fade; fBm sums octaves of doubling
// frequency and halving amplitude, normalised to [-1, 1].
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "../../include/libsvo_b200.h"

namespace {

uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double lattice(int64_t x, int64_t y, int64_t z, uint64_t seed) {
  const uint64_t h = mix64(seed ^ ((uint64_t)x * 0x8CB92BA72F3D8DD7ull) ^
                           ((uint64_t)y * 0xC13FA9A902A6328Full) ^ ((uint64_t)z * 0x91E10DA5C79E7B1Dull));
  return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

double fade(double t) { return t * t * (3.0 - 2.0 * t); }

double value_noise3(double x, double y, double z, uint64_t seed) {
  const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  const int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
  const double u = fade(x - fx), v = fade(y - fy), w = fade(z - fz);
  double c[2][2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
  const double x00 = c[0][0][0] + u * (c[1][0][0] - c[0][0][0]);
  const double x10 = c[0][1][0] + u * (c[1][1][0] - c[0][1][0]);
  const double x01 = c[0][0][1] + u * (c[1][0][1] - c[0][0][1]);
  const double x11 = c[0][1][1] + u * (c[1][1][1] - c[0][1][1]);
  const double y0 = x00 + v * (x10 - x00);
  const double y1 = x01 + v * (x11 - x01);
  return y0 + w * (y1 - y0);
}

double fbm3(double x, double y, double z, uint32_t octaves, double freq, uint64_t seed) {
  double sum = 0.0, amp = 1.0, norm = 0.0;
  for (uint32_t o = 0; o < octaves; ++o) {
    sum += amp * value_noise3(x * freq, y * freq, z * freq, seed + 0x1000193ull * (o + 1));
    norm += amp;
    amp *= 0.5;
    freq *= 2.0;
  }
  return norm > 0.0 ? sum / norm : 0.0;
}

}  // namespace

extern "C" {

int svo_mesh_icosphere_size(uint32_t subdivisions, uint64_t* num_vertices, uint64_t* num_triangles) {
  if (subdivisions > 11) return SVO_ERR_RANGE;
  const uint64_t p = 1ull << (2 * subdivisions);
  if (num_vertices) *num_vertices = 10 * p + 2;
  if (num_triangles) *num_triangles = 20 * p;
  return SVO_OK;
}

int svo_mesh_icosphere(uint32_t subdivisions, float radius, uint32_t octaves, float amplitude,
                       float frequency, uint64_t seed, float* h_vertices, uint32_t* h_triangles) {
  if (!h_vertices || !h_triangles) return SVO_ERR_INVALID;
  uint64_t nv_final = 0, nt_final = 0;
  int rc = svo_mesh_icosphere_size(subdivisions, &nv_final, &nt_final);
  if (rc != SVO_OK) return rc;
  try {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<double> v = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
                             0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
    std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                               11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                               3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (uint32_t s = 0; s < subdivisions; ++s) {
      std::unordered_map<uint64_t, uint32_t> mid;
      mid.reserve(f.size());
      std::vector<uint32_t> nf;
      nf.reserve(f.size() * 4);
      auto midpoint = [&](uint32_t a, uint32_t b) {
        const uint64_t key = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
        auto it = mid.find(key);
        if (it != mid.end()) return it->second;
        const uint32_t id = (uint32_t)(v.size() / 3);
        for (int k = 0; k < 3; ++k) v.push_back(0.5 * (v[3 * a + k] + v[3 * b + k]));
        mid.emplace(key, id);
        return id;
      };
      for (size_t i = 0; i < f.size(); i += 3) {
        const uint32_t a = f[i], b = f[i + 1], c = f[i + 2];
        const uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
        const uint32_t tri[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
        nf.insert(nf.end(), tri, tri + 12);
      }
      f.swap(nf);
    }
    if (v.size() / 3 != nv_final || f.size() / 3 != nt_final) return SVO_ERR_INVALID;
    for (uint64_t i = 0; i < nv_final; ++i) {
      double x = v[3 * i], y = v[3 * i + 1], z = v[3 * i + 2];
      const double l = std::sqrt(x * x + y * y + z * z);
      x /= l;
      y /= l;
      z /= l;
      const double r = radius + amplitude * fbm3(x, y, z, octaves, frequency, seed);
      h_vertices[3 * i] = (float)(x * r);
      h_vertices[3 * i + 1] = (float)(y * r);
      h_vertices[3 * i + 2] = (float)(z * r);
    }
    for (uint64_t i = 0; i < f.size(); ++i) h_triangles[i] = f[i];
  } catch (...) {
    return SVO_ERR_NOMEM;
  }
  return SVO_OK;
}

int svo_mesh_terrain_size(uint32_t grid, uint64_t* num_vertices, uint64_t* num_triangles) {
  if (grid < 2 || grid > 16384) return SVO_ERR_RANGE;
  if (num_vertices) *num_vertices = (uint64_t)grid * grid;
  if (num_triangles) *num_triangles = 2ull * (grid - 1) * (grid - 1);
  return SVO_OK;
}

int svo_mesh_terrain(uint32_t grid, uint32_t octaves, float base, float height, float frequency,
                     uint64_t seed, float* h_vertices, uint32_t* h_triangles) {
  if (!h_vertices || !h_triangles) return SVO_ERR_INVALID;
  int rc = svo_mesh_terrain_size(grid, nullptr, nullptr);
  if (rc != SVO_OK) return rc;
  const double step = 1.0 / (double)(grid - 1);
  for (uint32_t j = 0; j < grid; ++j)
    for (uint32_t i = 0; i < grid; ++i) {
      const double x = -0.5 + i * step, z = -0.5 + j * step;
      const double h01 = 0.5 * (fbm3(x, 0.0, z, octaves, frequency, seed) + 1.0);
      float* p = h_vertices + 3 * ((uint64_t)j * grid + i);
      p[0] = (float)x;
      p[1] = (float)(base + height * h01);
      p[2] = (float)z;
    }
  uint64_t k = 0;
  for (uint32_t j = 0; j + 1 < grid; ++j)
    for (uint32_t i = 0; i + 1 < grid; ++i) {
      const uint32_t a = j * grid + i, b = a + 1, c = a + grid, d = c + 1;
      const uint32_t tri[6] = {a, c, b, b, c, d};
      for (int q = 0; q < 6; ++q) h_triangles[k++] = tri[q];
    }
  return SVO_OK;
}

// Vertex normals: the normalised sum of the adjacent faces' cross products
// (area weighted), in double.  Vertex colours: three seeded value-noise
// fields of the position (frequency 3), mapped from [-1, 1] to [0.15, 0.95].
int svo_mesh_vertex_attributes(const float* h_vertices, uint64_t num_vertices,
                               const uint32_t* h_triangles, uint64_t num_triangles, uint64_t seed,
                               float* h_normals, float* h_colors) {
  if (!h_vertices || !h_triangles || !h_normals || !h_colors) return SVO_ERR_INVALID;
  for (uint64_t i = 0; i < 3 * num_triangles; ++i)
    if (h_triangles[i] >= num_vertices) return SVO_ERR_INVALID;
  try {
    std::vector<double> acc(3 * num_vertices, 0.0);
    for (uint64_t t = 0; t < num_triangles; ++t) {
      const uint32_t* f = h_triangles + 3 * t;
      const float* a = h_vertices + 3 * (uint64_t)f[0];
      const float* b = h_vertices + 3 * (uint64_t)f[1];
      const float* c = h_vertices + 3 * (uint64_t)f[2];
      const double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
      const double e2[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
      const double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                           e1[0] * e2[1] - e1[1] * e2[0]};
      for (int q = 0; q < 3; ++q)
        for (int k = 0; k < 3; ++k) acc[3 * (uint64_t)f[q] + k] += n[k];
    }
    for (uint64_t i = 0; i < num_vertices; ++i) {
      const double* n = &acc[3 * i];
      const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      for (int k = 0; k < 3; ++k) h_normals[3 * i + k] = l > 0.0 ? (float)(n[k] / l) : (k == 2 ? 1.0f : 0.0f);
      const float* p = h_vertices + 3 * i;
      for (int k = 0; k < 3; ++k) {
        const double f = value_noise3(3.0 * p[0], 3.0 * p[1], 3.0 * p[2], seed + 0x51ED27ull * (k + 1));
        h_colors[3 * i + k] = (float)(0.55 + 0.4 * f);
      }
    }
  } catch (...) {
    return SVO_ERR_NOMEM;
  }
  return SVO_OK;
}

}  // extern "C"
