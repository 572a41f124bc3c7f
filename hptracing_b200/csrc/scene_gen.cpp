// Seeded synthetic scenes used by the tests and benchmarks (the reference
// renders OBJ files; these stand in for them with the same array formats):
//   0  box room: open-front unit room, coloured side walls, an emissive
//      0.25 x 0.25 quad under the ceiling (Ke 15), a diffuse 0.3x0.6x0.3 box
//      and a glass 0.3^3 box (ior 1.5) rotated +-17 degrees about y.
//   1  room + 64 UV spheres (32 x 16 segments, 960 triangles each), 60 %
//      diffuse, 20 % mirror, 20 % glass; half carry value-noise textures
//      (1024^2 RGBA8 nominal) with spherical UVs.
//   2  1024 x 1024-vertex fractal value-noise heightfield (6 octaves,
//      amplitude 0.15, interpolated normals) + 16 columns of 20k triangles,
//      8 value-noise textures (2048^2 nominal) with planar UVs, a 2 x 2
//      emissive quad (Ke 10) overhead.
//   3  a family-0/1/2 scene tessellated to about target_triangles.
// Every quad is emitted as the fan (v0,v1,v2), (v0,v2,v3) that the OBJ
// reader produces, so no emissive triangle has its right angle at v0 (the
// reference's light-area formula divides by the cosine at v0).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "host.h"

namespace hpt {

namespace {

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  double uniform() { return (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
};

// Value noise on an integer lattice with a smoothstep blend.
struct ValueNoise {
  uint64_t seed;
  float lattice(int64_t x, int64_t y) const {
    uint64_t s = seed ^ ((uint64_t)x * 0x8CB92BA72F3D8DD7ull) ^ ((uint64_t)y * 0x9E3779B97F4A7C15ull);
    return (float)((splitmix(s) >> 40) * (1.0 / 16777216.0));
  }
  float at(double x, double y) const {
    double fx = std::floor(x), fy = std::floor(y);
    int64_t ix = (int64_t)fx, iy = (int64_t)fy;
    double tx = x - fx, ty = y - fy;
    tx = tx * tx * (3 - 2 * tx);
    ty = ty * ty * (3 - 2 * ty);
    double a = lattice(ix, iy), b = lattice(ix + 1, iy);
    double c = lattice(ix, iy + 1), d = lattice(ix + 1, iy + 1);
    return (float)((a + (b - a) * tx) + ((c + (d - c) * tx) - (a + (b - a) * tx)) * ty);
  }
  float fbm(double x, double y, int octaves) const {
    double sum = 0, amp = 0.5, freq = 1;
    for (int o = 0; o < octaves; ++o) {
      sum += amp * (at(x * freq + o * 17.31, y * freq - o * 9.71) - 0.5);
      amp *= 0.5;
      freq *= 2;
    }
    return (float)sum;
  }
};

// Runs f(row) for rows [0, n) on all host cores.
template <typename F>
void parallel_rows(int n, F&& f) {
  const int workers = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()),
                                              (unsigned)std::max(1, n));
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  auto run = [&] {
    for (int r = next++; r < n; r = next++) f(r);
  };
  for (int w = 1; w < workers; ++w) th.emplace_back(run);
  run();
  for (std::thread& t : th) t.join();
}

struct V3 {
  double x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
V3 normalized(V3 a) {
  double n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return n > 0 ? a * (1.0 / n) : a;
}

struct Builder {
  Mesh& m;
  explicit Builder(Mesh& mesh) : m(mesh) {}

  int material(const float kd[3], const float ke[3], const float ks[3],
               float dissolve, float ior, float ns, int diffuse_tex = -1) {
    hpt_ref_material x;
    memset(&x, 0, sizeof x);
    for (int k = 0; k < 3; ++k) {
      x.diffuse[k] = kd[k];
      x.emission[k] = ke[k];
      x.specular[k] = ks[k];
    }
    x.dissolve = dissolve;
    x.optical_density = ior;
    x.shininess = ns;
    x.diffuse_texture_id = diffuse_tex;
    x.ambient_texture_id = -1;
    material_probabilities(x);
    m.materials.push_back(x);
    return (int)m.materials.size() - 1;
  }
  int diffuse(float r, float g, float b, int tex = -1) {
    const float kd[3] = {r, g, b}, z[3] = {0, 0, 0};
    return material(kd, z, z, 1.f, 1.f, 1.f, tex);
  }
  int vertex(V3 p, V3 n, double u, double v) {
    m.points.push_back({(float)p.x, (float)p.y, (float)p.z, 0.f});
    m.normals.push_back({(float)n.x, (float)n.y, (float)n.z, 0.f});
    m.texcoords.push_back({(float)u, (float)v});
    return (int)m.points.size() - 1;
  }
  void tri(int a, int b, int c, int mat) { m.triangles.push_back({a, b, c, mat}); }
  // Quad p0..p3 (counter-clockwise) with a flat normal, split as a fan.
  void quad(V3 p0, V3 p1, V3 p2, V3 p3, V3 n, int mat) {
    int a = vertex(p0, n, 0, 0), b = vertex(p1, n, 1, 0);
    int c = vertex(p2, n, 1, 1), d = vertex(p3, n, 0, 1);
    tri(a, b, c, mat);
    tri(a, c, d, mat);
  }
  // Grid-tessellated quad (k x k cells): origin + s*du + t*dv.
  void grid(V3 origin, V3 du, V3 dv, V3 n, int k, int mat) {
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        double s0 = (double)j / k, s1 = (double)(j + 1) / k;
        double t0 = (double)i / k, t1 = (double)(i + 1) / k;
        quad(origin + du * s0 + dv * t0, origin + du * s1 + dv * t0,
             origin + du * s1 + dv * t1, origin + du * s0 + dv * t1, n, mat);
      }
  }
  // Box of size (sx, sy, sz) standing on y = y0, centred at (cx, cz),
  // rotated by `deg` about the vertical axis; 6 faces, 12 triangles.
  void box(double cx, double y0, double cz, double sx, double sy, double sz,
           double deg, int mat) {
    double a = deg * M_PI / 180.0, ca = std::cos(a), sa = std::sin(a);
    auto P = [&](double x, double y, double z) {
      double lx = x * sx - sx / 2, lz = z * sz - sz / 2;
      return V3{cx + ca * lx + sa * lz, y0 + y * sy, cz - sa * lx + ca * lz};
    };
    auto R = [&](V3 n) { return V3{ca * n.x + sa * n.z, n.y, -sa * n.x + ca * n.z}; };
    quad(P(0, 0, 0), P(0, 0, 1), P(1, 0, 1), P(1, 0, 0), V3{0, -1, 0}, mat);
    quad(P(0, 1, 0), P(1, 1, 0), P(1, 1, 1), P(0, 1, 1), V3{0, 1, 0}, mat);
    quad(P(0, 0, 0), P(1, 0, 0), P(1, 1, 0), P(0, 1, 0), R(V3{0, 0, -1}), mat);
    quad(P(0, 0, 1), P(0, 1, 1), P(1, 1, 1), P(1, 0, 1), R(V3{0, 0, 1}), mat);
    quad(P(0, 0, 0), P(0, 1, 0), P(0, 1, 1), P(0, 0, 1), R(V3{-1, 0, 0}), mat);
    quad(P(1, 0, 0), P(1, 0, 1), P(1, 1, 1), P(1, 1, 0), R(V3{1, 0, 0}), mat);
  }
  // UV sphere: `seg` longitudes x `rings` latitudes, spherical UVs; the pole
  // bands are single triangles (seg*2 + seg*(rings-2)*2 triangles).
  void sphere(V3 c, double r, int seg, int rings, int mat) {
    int base = (int)m.points.size();
    for (int i = 0; i <= rings; ++i) {
      double th = M_PI * i / rings;
      for (int j = 0; j <= seg; ++j) {
        double ph = 2 * M_PI * j / seg;
        V3 n{std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph)};
        vertex(c + n * r, n, (double)j / seg, (double)i / rings);
      }
    }
    auto id = [&](int i, int j) { return base + i * (seg + 1) + j; };
    for (int i = 0; i < rings; ++i)
      for (int j = 0; j < seg; ++j) {
        int a = id(i, j), b = id(i, j + 1), cc = id(i + 1, j + 1), d = id(i + 1, j);
        if (i == 0) {
          tri(a, cc, d, mat);
        } else if (i == rings - 1) {
          tri(a, b, cc, mat);
        } else {
          tri(a, b, cc, mat);
          tri(a, cc, d, mat);
        }
      }
  }
  // Vertical cylinder side (no caps): seg x stacks quads.
  void column(V3 base_c, double r, double h, int seg, int stacks, int mat) {
    int base = (int)m.points.size();
    for (int i = 0; i <= stacks; ++i)
      for (int j = 0; j <= seg; ++j) {
        double ph = 2 * M_PI * j / seg;
        V3 n{std::cos(ph), 0, std::sin(ph)};
        V3 p = base_c + V3{0, h * i / stacks, 0} + n * r;
        vertex(p, n, (double)j / seg, (double)i / stacks);
      }
    auto id = [&](int i, int j) { return base + i * (seg + 1) + j; };
    for (int i = 0; i < stacks; ++i)
      for (int j = 0; j < seg; ++j) {
        tri(id(i, j), id(i, j + 1), id(i + 1, j + 1), mat);
        tri(id(i, j), id(i + 1, j + 1), id(i + 1, j), mat);
      }
  }
  void texture(int size, uint64_t seed) {
    ValueNoise n{seed};
    ValueNoise n2{seed * 7 + 3};
    m.texture_dims.push_back(size);
    m.texture_dims.push_back(size);
    size_t off = m.texture_data.size();
    m.texture_data.resize(off + (size_t)size * size * 4);
    uint8_t* dst = m.texture_data.data() + off;
    float c0[3] = {(float)((seed >> 3) % 7) / 7.f, 0.5f, 0.9f};
    // Every texel is a pure function of (x, y): rows are filled in parallel.
    parallel_rows(size, [&](int y) {
      for (int x = 0; x < size; ++x) {
        double u = 16.0 * x / size, v = 16.0 * y / size;
        float a = 0.5f + n.fbm(u, v, 4), b = 0.5f + n2.fbm(u * 2, v * 2, 3);
        uint8_t* px = dst + ((size_t)y * size + x) * 4;
        for (int k = 0; k < 3; ++k) {
          float val = 0.15f + 0.8f * (k == 0 ? a : k == 1 ? 0.5f * (a + b) : b) * (0.6f + 0.4f * c0[k]);
          px[k] = (uint8_t)std::min(255.f, std::max(0.f, val * 255.f));
        }
        px[3] = 0;
      }
    });
    m.texture_names.push_back("noise" + std::to_string(m.texture_names.size()));
  }
};

// Box room (config 0). wall_k tessellates each wall into k x k cells.
void room(Builder& b, int wall_k, int box_k) {
  int white = b.diffuse(0.75f, 0.75f, 0.75f);
  int red = b.diffuse(0.75f, 0.25f, 0.25f);
  int green = b.diffuse(0.25f, 0.75f, 0.25f);
  const float z3[3] = {0, 0, 0}, ke[3] = {15, 15, 15};
  int light = b.material(z3, ke, z3, 1.f, 1.f, 1.f);
  int boxmat = b.diffuse(0.75f, 0.75f, 0.75f);
  const float ks0[3] = {0, 0, 0};
  int glass = b.material(z3, z3, ks0, 0.f, 1.5f, 1.f);
  b.grid(V3{0, 0, 0}, V3{1, 0, 0}, V3{0, 0, 1}, V3{0, 1, 0}, wall_k, white);   // floor
  b.grid(V3{0, 1, 0}, V3{0, 0, 1}, V3{1, 0, 0}, V3{0, -1, 0}, wall_k, white);  // ceiling
  b.grid(V3{0, 0, 1}, V3{0, 1, 0}, V3{1, 0, 0}, V3{0, 0, -1}, wall_k, white);  // back
  b.grid(V3{0, 0, 0}, V3{0, 0, 1}, V3{0, 1, 0}, V3{1, 0, 0}, wall_k, red);     // left
  b.grid(V3{1, 0, 0}, V3{0, 1, 0}, V3{0, 0, 1}, V3{-1, 0, 0}, wall_k, green);  // right
  b.quad(V3{0.375, 0.999, 0.375}, V3{0.625, 0.999, 0.375}, V3{0.625, 0.999, 0.625},
         V3{0.375, 0.999, 0.625}, V3{0, -1, 0}, light);
  (void)box_k;
  b.box(0.34, 0.0, 0.64, 0.3, 0.6, 0.3, 17.0, boxmat);
  b.box(0.66, 0.0, 0.34, 0.3, 0.3, 0.3, -17.0, glass);
}

void spheres(Builder& b, Rng& rng, int count, int seg, int rings, int tex_size,
             uint64_t seed) {
  int ntex = tex_size > 0 ? 4 : 0;
  int tex_base = (int)b.m.texture_names.size();
  for (int t = 0; t < ntex; ++t) b.texture(tex_size, seed * 131 + t);
  for (int i = 0; i < count; ++i) {
    V3 c{rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9)};
    double r = rng.uniform(0.04, 0.12);
    double kind = rng.uniform();
    int tex = (ntex && (i % 2 == 0)) ? tex_base + (i / 2) % ntex : -1;
    int mat;
    const float z3[3] = {0, 0, 0};
    if (kind < 0.6) {
      mat = b.diffuse((float)rng.uniform(0.2, 0.9), (float)rng.uniform(0.2, 0.9),
                      (float)rng.uniform(0.2, 0.9), tex);
    } else if (kind < 0.8) {
      const float ks[3] = {1, 1, 1};
      mat = b.material(z3, z3, ks, 1.f, 1.f, 1000.f, tex);
    } else {
      mat = b.material(z3, z3, z3, 0.f, 1.5f, 1.f, tex);
    }
    b.sphere(c, r, seg, rings, mat);
  }
}

void terrain(Builder& b, Rng& rng, int n, int tex_size, int ntex,
             int col_seg, int col_stacks, uint64_t seed) {
  ValueNoise noise{seed ^ 0x5A5A5A5Aull};
  int tex_base = (int)b.m.texture_names.size();
  for (int t = 0; t < ntex; ++t) b.texture(tex_size, seed * 977 + t);
  std::vector<int> mats;
  for (int t = 0; t < std::max(ntex, 1); ++t)
    mats.push_back(b.diffuse(0.8f, 0.8f, 0.8f, ntex ? tex_base + t : -1));
  auto height = [&](double x, double z) { return 0.15 * noise.fbm(x * 2.5 + 7, z * 2.5 + 3, 6); };
  int base = (int)b.m.points.size();
  double h = 2.0 / (n - 1);
  // Heights and normals are pure functions of the grid point: computed in
  // parallel by rows, appended in row order.
  std::vector<V3> pos((size_t)n * n), nrm((size_t)n * n);
  parallel_rows(n, [&](int i) {
    for (int j = 0; j < n; ++j) {
      double x = -1 + j * h, z = -1 + i * h;
      double y = height(x, z);
      double dx = (height(x + h, z) - height(x - h, z)) / (2 * h);
      double dz = (height(x, z + h) - height(x, z - h)) / (2 * h);
      pos[(size_t)i * n + j] = V3{x, y, z};
      nrm[(size_t)i * n + j] = normalized(V3{-dx, 1, -dz});
    }
  });
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const V3& p = pos[(size_t)i * n + j];
      b.vertex(p, nrm[(size_t)i * n + j], (p.x + 1) * 2, (p.z + 1) * 2);
    }
  for (int i = 0; i + 1 < n; ++i)
    for (int j = 0; j + 1 < n; ++j) {
      int a = base + i * n + j, c = base + (i + 1) * n + j + 1;
      int bb = base + i * n + j + 1, d = base + (i + 1) * n + j;
      int mat = mats[(j * (int)mats.size()) / (n - 1)];
      b.tri(a, bb, c, mat);
      b.tri(a, c, d, mat);
    }
  const float z3[3] = {0, 0, 0};
  int colmat = b.diffuse(0.7f, 0.7f, 0.65f);
  const float ks[3] = {0.9f, 0.9f, 0.9f};
  int colmirror = b.material(z3, z3, ks, 1.f, 1.f, 500.f);
  for (int k = 0; k < 16; ++k) {
    double cx = -0.75 + 0.5 * (k % 4), cz = -0.75 + 0.5 * (k / 4);
    double y0 = height(cx, cz) - 0.05;
    b.column(V3{cx, y0, cz}, 0.05 + 0.02 * rng.uniform(), 0.5 + 0.3 * rng.uniform(),
             col_seg, col_stacks, (k % 3 == 0) ? colmirror : colmat);
  }
  const float ke[3] = {10, 10, 10};
  int light = b.material(z3, ke, z3, 1.f, 1.f, 1.f);
  b.quad(V3{-1, 1.2, -1}, V3{1, 1.2, -1}, V3{1, 1.2, 1}, V3{-1, 1.2, 1}, V3{0, -1, 0}, light);
}

}  // namespace

hpt_status generate_scene(int config, uint64_t seed, const hpt_gen_params& p,
                          Mesh& out) {
  out = Mesh();
  Builder b(out);
  Rng rng(seed ^ 0x48505400ull);
  switch (config) {
    case 0:
      room(b, 1, 1);
      break;
    case 1:
      room(b, 1, 1);
      spheres(b, rng, 64, 32, 16, p.texture_size > 0 ? p.texture_size : 1024, seed);
      break;
    case 2: {
      int n = p.heightfield_n > 1 ? p.heightfield_n : 1024;
      int ts = p.texture_size > 0 ? p.texture_size : 2048;
      terrain(b, rng, n, ts, 8, 100, 100, seed);
      break;
    }
    case 3: {
      int target = std::max(40, p.target_triangles);
      int ts = p.texture_size > 0 ? p.texture_size : 256;
      if (p.family == 0) {
        // Room walls tessellated to reach the triangle budget.
        int k = std::max(1, (int)std::lround(std::sqrt(std::max(0, target - 26) / 10.0)));
        room(b, k, 1);
      } else if (p.family == 1) {
        room(b, 1, 1);
        // 64 spheres; choose the ring count so 64 * 2 * seg * (rings-1) ~ target.
        int rings = std::max(3, (int)std::lround(std::sqrt(std::max(64, target) / 256.0)));
        int seg = 2 * rings;
        spheres(b, rng, 64, seg, rings, ts, seed);
      } else {
        int n = std::max(3, (int)std::lround(std::sqrt(std::max(0, target - 16 * 200) / 2.0)) + 1);
        int cs = std::max(3, (int)std::lround(std::sqrt(std::max(200, target / 128) / 2.0)));
        terrain(b, rng, n, ts, 2, cs, cs, seed);
      }
      break;
    }
    default:
      return fail(HPT_ERR_INVALID_ARGUMENT, "unknown scene config %d", config);
  }
  if (!build_light_table(out.points, out.triangles, out.materials, out.lights))
    return fail(HPT_ERR_INVALID_SCENE, "light table: bad material index");
  return HPT_OK;
}

}  // namespace hpt
