// hpt_oracle.cpp - CPU restatement of the reference's wavefront path, used
// ONLY as the checker by tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py. Nothing in the product links it.
//
// It restates, in plain C++ (IEEE single precision, -ffp-contract=off):
//   - the kernels of src/hp/cl_src/kernel.cl (cited per function), with the
//     OpenCL vector built-ins expanded as
//       dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z, cross the usual way,
//       length = sqrt(dot(a,a)), normalize = a / length(a);
//   - read_imagef with CLK_NORMALIZED_COORDS_TRUE | CLK_ADDRESS_REPEAT |
//     CLK_FILTER_LINEAR on RGBA UNORM_INT8 per the OpenCL 1.2 specification;
//   - the host loop of TraceRunner::run (src/hp/trace_runner.cpp:116-356),
//     including the primary pass run once with sample_n = sample, the
//     per-lane LCG state v_seed[global_id] and the per-stage lists;
//   - an FP64 brute-force ray/triangle intersector for error statements.
// Parity is pinned by tests against the reference's own kernel.cl compiled
// as C++ (oracle/refcl, built into oracle/_ref/ when the reference sources
// are present) and against golden vectors under tests/golden/.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <random>
#include <thread>
#include <vector>

namespace {

struct V3 {
  float x, y, z;
};
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { return a / length(a); }

struct Node {  // KDTreeNodeHeader, types.h.cl:36-43
  float box_start[4], box_end[4];
  int32_t child, parent, sibling, data;
};
struct Material {  // types.h.cl:19-34
  float emission[4], ambient[4], diffuse[4], specular[4];
  float optical_density, dissolve, shininess;
  int32_t diffuse_texture_id, ambient_texture_id;
  float specular_possibility, refract_possibility, diffuse_possibility;
};
static_assert(sizeof(Node) == 48 && sizeof(Material) == 96, "reference layouts");

inline V3 f4(const float* p, int i) { return v3(p[4 * i], p[4 * i + 1], p[4 * i + 2]); }
inline V3 m3(const float* p) { return v3(p[0], p[1], p[2]); }

}  // namespace

extern "C" {

// Scene as seen by the kernels (the buffers TraceRunner uploads,
// trace_runner.cpp:65-86), plus per-texture dims.
struct OracleScene {
  const float* points;      // float4
  const float* normals;     // float4 or null
  int32_t num_normals;
  const float* texcoords;   // float2 or null
  int32_t num_texcoords;
  const int32_t* triangles; // int4
  int32_t num_triangles;
  const void* nodes;        // Node[]
  int32_t num_nodes;
  const int32_t* leaf_data;
  const void* materials;    // Material[]
  const int32_t* lights;    // int4
  int32_t num_lights;
  const uint8_t* texture_data;
  int32_t num_textures;
  const int32_t* texture_dims;  // (w, h) per texture
};

struct OracleCamera {
  float view_p[3], top_dir[3], right_dir[3];
  float width, height;
};

}  // extern "C"

namespace {

// ---- kernel.cl:26-47 -------------------------------------------------------
inline uint32_t lcg_rand(int64_t* seed) {
  *seed = (int64_t)(((uint64_t)*seed * 0x5DEECE66Dull + 0xBull) & ((1ull << 48) - 1));
  return (uint32_t)((*seed >> 16) & 0xFFFFFFFFll);
}
inline float lcg_randf(int64_t* seed) {
  return (float)lcg_rand(seed) / (float)0xFFFFFFFFll;
}
const float PI = 3.1415926535f;
inline V3 randf3(int64_t* seed) {
  float alpha = lcg_randf(seed) * PI;
  float beta = lcg_randf(seed) * PI;
  float cos_beta = std::cos(beta);
  return v3(cos_beta * std::cos(alpha), cos_beta * std::sin(alpha), std::sin(beta));
}

// ---- kernel.cl:51-83 -------------------------------------------------------
bool box_intersect(const float* bs, const float* be, V3 p, V3 d) {
  if (p.x >= bs[0] && p.x <= be[0] && p.y >= bs[1] && p.y <= be[1] && p.z >= bs[2] &&
      p.z <= be[2])
    return true;
  const float o[3] = {p.x, p.y, p.z}, dd[3] = {d.x, d.y, d.z};
  float mins[3], maxs[3];
  for (int a = 0; a < 3; ++a) {
    float t0 = (bs[a] - o[a]) / dd[a];
    float t1 = (be[a] - o[a]) / dd[a];
    mins[a] = std::fmin(t0, t1);
    maxs[a] = std::fmax(t0, t1);
  }
  float max_of_mins = std::fmax(std::fmax(mins[0], mins[1]), mins[2]);
  float min_of_maxs = std::fmin(std::fmin(maxs[0], maxs[1]), maxs[2]);
  if (min_of_maxs <= 0) return false;
  return max_of_mins <= min_of_maxs;
}

// ---- kernel.cl:85-109 (u, v reported as well) ------------------------------
float single_intersect(V3 start_p, V3 in_dir, V3 pa, V3 pb, V3 pc, float* uo, float* vo) {
  V3 e1 = pb - pa;
  V3 e2 = pc - pa;
  V3 P = cross(in_dir, e2);
  float det = dot(e1, P);
  float inv_det = 1.f / det;
  V3 T = start_p - pa;
  float u = dot(T, P) * inv_det;
  if (u < 0.f || u > 1.f) return -1;
  V3 Q = cross(T, e1);
  float v = dot(in_dir, Q) * inv_det;
  if (v < 0.f || u + v > 1.f) return -1;
  float t = dot(e2, Q) * inv_det;
  *uo = u;
  *vo = v;
  if (t > 0) return t;
  return -1;
}

struct IsectResult {
  int tri;
  float t, u, v;
  int leaves;     // leaves gathered (before the cap)
  int overflow;   // more than 512 leaves pierced
};

// ---- kernel.cl:111-192 -----------------------------------------------------
IsectResult kdtree_intersect(const OracleScene& s, V3 o, V3 d) {
  const Node* nodes = static_cast<const Node*>(s.nodes);
  int match[512];
  int nmatch = 0, pierced = 0;
  int node_index = 0, come_from_child = 0;
  int64_t guard = 0;
  while (true) {
    if (++guard > 64ll * s.num_nodes + 64) break;  // malformed-tree guard
    int goto_child = 0;
    const Node& node = nodes[node_index];
    if (come_from_child == 0 && box_intersect(node.box_start, node.box_end, o, d)) {
      if (node.child < 0) {
        if (node.data >= 0) {
          ++pierced;
          if (nmatch < 512) match[nmatch++] = node.data;
        }
      } else {
        goto_child = 1;
      }
    }
    if (goto_child) {
      come_from_child = 0;
      node_index = node.child;
    } else if (node.sibling >= 0) {
      come_from_child = 0;
      node_index = node.sibling;
    } else if (node.parent >= 0) {
      come_from_child = 1;
      node_index = node.parent;
    } else {
      break;
    }
  }
  IsectResult r{-1, -42.f, 0.f, 0.f, pierced, pierced > 512 ? 1 : 0};
  for (int i = 0; i < nmatch; ++i) {
    const int32_t* data = s.leaf_data + match[i];
    int n = data[0];
    for (int x = 0; x < n; ++x) {
      int id = data[x + 1];
      const int32_t* t4 = s.triangles + 4 * id;
      float u, v;
      float res = single_intersect(o, d, f4(s.points, t4[0]), f4(s.points, t4[1]),
                                   f4(s.points, t4[2]), &u, &v);
      if (res > 0 && (r.t < 0 || res < r.t)) {
        r.t = res;
        r.tri = id;
        r.u = u;
        r.v = v;
      }
    }
  }
  if (r.tri < 0) r.t = 0.f;
  return r;
}

// ---- read_imagef, OpenCL 1.2 spec (normalized, repeat, linear) -------------
V3 sample_texture(const OracleScene& s, int tex, float su, float sv) {
  if (tex < 0 || tex >= s.num_textures) return v3(0, 0, 0);
  int64_t off = 0;
  for (int k = 0; k < tex; ++k) off += (int64_t)s.texture_dims[2 * k] * s.texture_dims[2 * k + 1];
  const int w = s.texture_dims[2 * tex], h = s.texture_dims[2 * tex + 1];
  if (!std::isfinite(su)) su = 0.f;
  if (!std::isfinite(sv)) sv = 0.f;
  float u = (su - std::floor(su)) * (float)w;
  float v = (sv - std::floor(sv)) * (float)h;
  float x = u - 0.5f, y = v - 0.5f;
  float fx = std::floor(x), fy = std::floor(y);
  int i0 = (int)fx, j0 = (int)fy;
  float a = x - fx, b = y - fy;
  int i1 = i0 + 1, j1 = j0 + 1;
  if (i0 < 0) i0 += w;
  if (j0 < 0) j0 += h;
  if (i1 > w - 1) i1 -= w;
  if (j1 > h - 1) j1 -= h;
  auto texel = [&](int i, int j) {
    const uint8_t* p = s.texture_data + 4 * (off + (int64_t)j * w + i);
    return v3((float)p[0] / 255.f, (float)p[1] / 255.f, (float)p[2] / 255.f);
  };
  V3 r = ((1.f - a) * (1.f - b)) * texel(i0, j0);
  r = r + (a * (1.f - b)) * texel(i1, j0);
  r = r + ((1.f - a) * b) * texel(i0, j1);
  r = r + (a * b) * texel(i1, j1);
  return r;
}

struct Rec {  // the fields of unit_data the kernels use (types.h.cl:8-17)
  int orig_id;
  V3 strength, start_p, in_dir;
  int tri;
  float t;
  V3 intersect_p, normal;
  float optical_density, shininess;
};

// ---- s1_run, kernel.cl:258-409 (one element) -------------------------------
// Returns the branch (-1 terminated, 0 refract, 1 specular, 2 diffuse,
// 3 light); contrib receives the value added to the ray's accumulator.
int s1_run(const OracleScene& s, Rec& rec, int disable_diffuse, int64_t* seed, V3* contrib) {
  const int32_t* g = s.triangles + 4 * rec.tri;
  const Material& mat = static_cast<const Material*>(s.materials)[g[3]];
  V3 ga = f4(s.points, g[0]), gb = f4(s.points, g[1]), gc = f4(s.points, g[2]);
  V3 ip = rec.start_p + rec.t * rec.in_dir;
  V3 f1 = ga - ip, f2 = gb - ip, f3 = gc - ip;
  float area_all = length(cross(gb - ga, gc - ga));
  float area1 = length(cross(f2, f3)) / area_all;
  float area2 = length(cross(f1, f3)) / area_all;
  float area3 = length(cross(f1, f2)) / area_all;
  V3 normal;
  if (s.num_normals == 0)
    normal = normalize(cross(gb - ga, gc - ga));
  else
    normal = area1 * f4(s.normals, g[0]) + area2 * f4(s.normals, g[1]) +
             area3 * f4(s.normals, g[2]);
  float uvx = 0, uvy = 0;
  if (mat.ambient_texture_id >= 0 || mat.diffuse_texture_id >= 0) {
    if (s.num_texcoords == 0) {
      float len = std::sqrt(ip.x * ip.x + ip.y * ip.y);
      uvx = ip.x / len;
      uvy = ip.y / len;
    } else {
      const float* tc = s.texcoords;
      uvx = area1 * tc[2 * g[0]] + area2 * tc[2 * g[1]] + area3 * tc[2 * g[2]];
      uvy = area1 * tc[2 * g[0] + 1] + area2 * tc[2 * g[1] + 1] + area3 * tc[2 * g[2] + 1];
    }
    uvy = 1.f - uvy;
  }
  V3 ambient = m3(mat.ambient);
  if (mat.ambient_texture_id >= 0) ambient = sample_texture(s, mat.ambient_texture_id, uvx, uvy);
  V3 result = rec.strength * (ambient + m3(mat.emission));
  result = std::fabs(dot(normal, rec.in_dir)) * result;
  *contrib = result;
  if (length(rec.strength) < 1e-4f) return -1;
  rec.intersect_p = ip;
  rec.normal = normal;
  float rn = lcg_randf(seed);
  if (rn < mat.specular_possibility) {
    rec.strength = rec.strength * m3(mat.specular);
    rec.shininess = mat.shininess;
    return 1;
  }
  if (rn < mat.refract_possibility) {
    rec.strength = (1.0f - mat.dissolve) * rec.strength;
    rec.optical_density = mat.optical_density;
    return 0;
  }
  V3 diffuse = m3(mat.diffuse);
  if (mat.diffuse_texture_id >= 0) diffuse = sample_texture(s, mat.diffuse_texture_id, uvx, uvy);
  rec.strength = rec.strength * diffuse;
  return (rn < mat.diffuse_possibility && disable_diffuse == 0) ? 2 : 3;
}

// ---- s2_*_run, kernel.cl:413-557 (one element) -----------------------------
// Returns 1 if the ray is appended to S0.
int s2_run(const OracleScene& s, int branch, Rec& rec, int64_t* seed) {
  const float STEP = 1e-5f;
  if (branch == 0) {  // :413-449
    float cos_alpha = dot(rec.in_dir, -rec.normal);
    float reverse = 1.0f;
    if (cos_alpha < 0) reverse = -1;
    float alpha = std::acos(cos_alpha);
    V3 p = cos_alpha * rec.normal;
    V3 q = normalize(rec.in_dir + p);
    float sin_beta = std::sin(alpha) * std::pow(rec.optical_density, -reverse);
    V3 dir;
    if (sin_beta <= 1.f) {
      float beta = std::asin(sin_beta);
      dir = (-reverse * std::cos(beta)) * rec.normal + sin_beta * q;
    } else {
      dir = rec.in_dir + p + p;
    }
    rec.start_p = rec.intersect_p + STEP * dir;
    rec.in_dir = dir;
    return 1;
  }
  if (branch == 1) {  // :451-478
    V3 rv = randf3(seed) / 2.0f / rec.shininess;
    float d_ = dot(rec.in_dir, rec.normal);
    V3 projection = d_ * rec.normal;
    V3 dir = rec.in_dir - 2.0f * projection;
    dir = dir + rv;
    rec.start_p = rec.intersect_p + STEP * dir;
    rec.in_dir = dir;
    return 1;
  }
  if (branch == 2) {  // :480-510
    bool front = dot(rec.in_dir, rec.normal) < 0;
    V3 p = randf3(seed);
    float dn = dot(p, rec.normal);
    if (dn < 0) {
      dn = -dn;
      if (front) p = -p;
    }
    rec.strength = dn * rec.strength;
    rec.start_p = rec.intersect_p + STEP * p;
    rec.in_dir = p;
    return 1;
  }
  if (branch == 3) {  // :512-557
    if (s.num_lights == 0) return 0;
    bool front = dot(rec.in_dir, rec.normal) < 0;
    int li = (int)((int64_t)lcg_rand(seed) % s.num_lights);
    const int32_t* L = s.lights + 4 * li;
    V3 pa = f4(s.points, L[0]), pb = f4(s.points, L[1]), pc = f4(s.points, L[2]);
    float rx = lcg_randf(seed), ry = lcg_randf(seed);
    if (rx + ry > 1) {
      rx = 1 - rx;
      ry = 1 - ry;
    }
    V3 point = pa + rx * (pb - pa) + ry * (pc - pa);
    V3 p = normalize(point - rec.intersect_p);
    float d_ = dot(p, rec.normal);
    if ((d_ > 0) == front) {
      rec.strength = std::fabs(d_) * rec.strength;
      rec.start_p = rec.intersect_p + STEP * p;
      rec.in_dir = p;
      return 1;
    }
    return 0;
  }
  return 0;
}

// ---- set_viewdirs / set_viewdirs_vr, kernel.cl:559-613 ---------------------
V3 pinhole(const OracleCamera& c, int x, int y, int nx, int ny) {
  V3 top = m3(c.top_dir), right = m3(c.right_dir);
  V3 nd = cross(top, right);
  nd = nd + ((float)y / (float)ny * c.height - c.height * 0.5f) * top;
  nd = nd + ((float)x / (float)nx * c.width - c.width * 0.5f) * right;
  return normalize(nd);
}
V3 pano(int x, int y, int x_shift, int sample_y) {
  float lon = (float)(x + x_shift) / (float)(sample_y * 2) * PI * 2 - PI;
  float lat = (float)((double)((float)y / (float)sample_y * PI) - (double)PI / 2.0);
  return normalize(v3(std::cos(lat) * std::cos(lon), std::sin(lat), std::cos(lat) * std::sin(lon)));
}

// Parallel for over [0, n) with up to `threads` workers.
void pfor(int64_t n, int threads, const std::function<void(int64_t, int64_t)>& f) {
  if (threads <= 1 || n < 256) {
    f(0, n);
    return;
  }
  std::vector<std::thread> ts;
  int64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    int64_t b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    ts.emplace_back(f, b, e);
  }
  for (auto& t : ts) t.join();
}

uint64_t path_seed(uint64_t key, uint32_t ray, uint32_t sample, uint32_t bounce) {
  uint64_t z = key ^ (((uint64_t)ray << 32) | sample) * 0x9E3779B97F4A7C15ull;
  z ^= (uint64_t)(bounce + 1) * 0xD1B54A32D192ED03ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z & ((1ull << 48) - 1);
}

}  // namespace

extern "C" {

// Stage entry points ---------------------------------------------------------

int oracle_box_intersect(const float* box_start, const float* box_end, const float* p,
                         const float* d) {
  return box_intersect(box_start, box_end, v3(p[0], p[1], p[2]), v3(d[0], d[1], d[2])) ? 1 : 0;
}

void oracle_intersect(const OracleScene* s, int n, const float* o, const float* d, int32_t* tri,
                      float* t, float* u, float* v, int32_t* leaves, int32_t* overflow,
                      int threads) {
  pfor(n, threads, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      IsectResult r = kdtree_intersect(*s, v3(o[3 * i], o[3 * i + 1], o[3 * i + 2]),
                                       v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
      tri[i] = r.tri;
      t[i] = r.t;
      u[i] = r.tri >= 0 ? r.u : 0.f;
      v[i] = r.tri >= 0 ? r.v : 0.f;
      if (leaves) leaves[i] = r.leaves;
      if (overflow) overflow[i] = r.overflow;
    }
  });
}

// FP64 brute force: closest positive t over all triangles (same formula).
void oracle_brute_f64(const OracleScene* s, int n, const float* o, const float* d, int32_t* tri,
                      double* t, int threads) {
  pfor(n, threads, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      double O[3] = {o[3 * i], o[3 * i + 1], o[3 * i + 2]};
      double D[3] = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
      double best = -1;
      int bt = -1;
      for (int k = 0; k < s->num_triangles; ++k) {
        const int32_t* g = s->triangles + 4 * k;
        double A[3], B[3], C[3];
        for (int a = 0; a < 3; ++a) {
          A[a] = s->points[4 * g[0] + a];
          B[a] = s->points[4 * g[1] + a];
          C[a] = s->points[4 * g[2] + a];
        }
        double e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
        double e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
        double P[3] = {D[1] * e2[2] - D[2] * e2[1], D[2] * e2[0] - D[0] * e2[2],
                       D[0] * e2[1] - D[1] * e2[0]};
        double det = e1[0] * P[0] + e1[1] * P[1] + e1[2] * P[2];
        if (det == 0) continue;
        double inv = 1.0 / det;
        double T[3] = {O[0] - A[0], O[1] - A[1], O[2] - A[2]};
        double u = (T[0] * P[0] + T[1] * P[1] + T[2] * P[2]) * inv;
        if (u < 0 || u > 1) continue;
        double Q[3] = {T[1] * e1[2] - T[2] * e1[1], T[2] * e1[0] - T[0] * e1[2],
                       T[0] * e1[1] - T[1] * e1[0]};
        double v = (D[0] * Q[0] + D[1] * Q[1] + D[2] * Q[2]) * inv;
        if (v < 0 || u + v > 1) continue;
        double tt = (e2[0] * Q[0] + e2[1] * Q[1] + e2[2] * Q[2]) * inv;
        if (tt > 0 && (best < 0 || tt < best)) {
          best = tt;
          bt = k;
        }
      }
      tri[i] = bt;
      t[i] = bt >= 0 ? best : 0.0;
    }
  });
}

// s1_run per element; seeds[i] is the LCG state element i draws from
// (the reference's v_seed[global_id] + global_id), updated in place.
void oracle_shade(const OracleScene* s, int n, const float* o, const float* d, const float* strength,
                  const int32_t* tri, const float* t, int64_t* seeds, int disable_diffuse,
                  float* contrib, int32_t* branch, float* hit_p, float* normal,
                  float* strength_out, float* param) {
  for (int i = 0; i < n; ++i) {
    Rec r;
    memset(&r, 0, sizeof r);
    r.start_p = v3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
    r.in_dir = v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
    r.strength = v3(strength[3 * i], strength[3 * i + 1], strength[3 * i + 2]);
    r.tri = tri[i];
    r.t = t[i];
    V3 c;
    int b = s1_run(*s, r, disable_diffuse, &seeds[i], &c);
    if (b < 0) {
      // terminated before the hit record is written (kernel.cl:351-352)
      V3 ip = r.start_p + r.t * r.in_dir;
      r.intersect_p = ip;
    }
    contrib[3 * i] = c.x; contrib[3 * i + 1] = c.y; contrib[3 * i + 2] = c.z;
    branch[i] = b;
    hit_p[3 * i] = r.intersect_p.x; hit_p[3 * i + 1] = r.intersect_p.y; hit_p[3 * i + 2] = r.intersect_p.z;
    normal[3 * i] = r.normal.x; normal[3 * i + 1] = r.normal.y; normal[3 * i + 2] = r.normal.z;
    strength_out[3 * i] = r.strength.x;
    strength_out[3 * i + 1] = r.strength.y;
    strength_out[3 * i + 2] = r.strength.z;
    param[i] = b == 1 ? r.shininess : (b == 0 ? r.optical_density : 0.f);
  }
}

void oracle_next_dir(const OracleScene* s, int n, const int32_t* branch, const float* d,
                     const float* hit_p, const float* normal, const float* strength,
                     const float* param, int64_t* seeds, float* o_out, float* d_out, float* s_out,
                     int32_t* alive) {
  for (int i = 0; i < n; ++i) {
    Rec r;
    memset(&r, 0, sizeof r);
    r.in_dir = v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
    r.intersect_p = v3(hit_p[3 * i], hit_p[3 * i + 1], hit_p[3 * i + 2]);
    r.start_p = r.intersect_p;
    r.normal = v3(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]);
    r.strength = v3(strength[3 * i], strength[3 * i + 1], strength[3 * i + 2]);
    r.shininess = param[i];
    r.optical_density = param[i];
    int a = s2_run(*s, branch[i], r, &seeds[i]);
    alive[i] = a;
    o_out[3 * i] = r.start_p.x; o_out[3 * i + 1] = r.start_p.y; o_out[3 * i + 2] = r.start_p.z;
    d_out[3 * i] = r.in_dir.x; d_out[3 * i + 1] = r.in_dir.y; d_out[3 * i + 2] = r.in_dir.z;
    s_out[3 * i] = r.strength.x; s_out[3 * i + 1] = r.strength.y; s_out[3 * i + 2] = r.strength.z;
  }
}

void oracle_raygen(const OracleCamera* c, int sample_x, int sample_y, int ssx, int ssy, float* o,
                   float* d) {
  // trace_runner.cpp:131-150
  const int nx = sample_x * ssx, ny = sample_y * ssy;
  const bool vr = c->height < 0;
  const int shift = (int)c->right_dir[0] * ssx;
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      int64_t idx = (int64_t)nx * y + x;
      V3 dir = vr ? pano(x, y, shift, ny) : pinhole(*c, x, y, nx, ny);
      o[3 * idx] = c->view_p[0]; o[3 * idx + 1] = c->view_p[1]; o[3 * idx + 2] = c->view_p[2];
      d[3 * idx] = dir.x; d[3 * idx + 1] = dir.y; d[3 * idx + 2] = dir.z;
    }
}

// get_image, kernel.cl:615-652; write_imagef RGBA UNORM_INT8 conversion is
// convert_uchar_sat_rte(x * 255).
void oracle_resolve(const float* accum, int W, int H, int ssx, int ssy, int sample,
                    float brightness, uint8_t* rgba) {
  for (int gy = 0; gy < H; ++gy)
    for (int gx = 0; gx < W; ++gx) {
      float p[4] = {0, 0, 0, 0};
      for (int i = 0; i < ssx; ++i)
        for (int j = 0; j < ssy; ++j) {
          int64_t idx = (int64_t)(gy * ssy + j) * W * ssx + gx * ssx + i;
          for (int c = 0; c < 3; ++c) p[c] += accum[3 * idx + c];
        }
      uint8_t* out = rgba + 4 * ((int64_t)gy * W + gx);
      for (int c = 0; c < 3; ++c) {
        float x = p[c] / (float)(ssx * ssy);
        x = x / (float)sample;
        x = x * brightness;
        x = 1.f - std::exp(-x);
        float v = x * 255.0f;
        out[c] = !(v >= 0.f) ? 0 : (v >= 255.f ? 255 : (uint8_t)std::nearbyint(v));
      }
      out[3] = 0;
    }
}

// TraceRunner::run (trace_runner.cpp:116-356) on host threads.
//   rng_mode 0: the reference's per-lane LCG state v_seed[global_id], seeded
//               from `seed` (the reference seeds from time(0));
//   rng_mode 1: the counter-based per-(ray, sample, bounce) streams of the
//               GPU path, so paths match the GPU's one for one.
// accum: 3 floats per ray; accum2 (nullable): per-ray sum over samples of
// the squared per-sample radiance, for Monte Carlo error bars.
// counts[0] = intersect queries, counts[1] = shade calls,
// counts[2] = rays whose gather exceeded 512 leaves.
void oracle_render(const OracleScene* s, const OracleCamera* cam, int sample_x, int sample_y,
                   int ssx, int ssy, const float* bg, int sample, int depth, int disable_diffuse,
                   uint64_t seed, int rng_mode, int threads, float* accum, float* accum2,
                   int64_t* counts) {
  const int nx = sample_x * ssx, ny = sample_y * ssy;
  const int64_t n = (int64_t)nx * ny;
  std::vector<float> o(3 * n), d(3 * n);
  oracle_raygen(cam, sample_x, sample_y, ssx, ssy, o.data(), d.data());
  std::vector<Rec> initial(n);
  for (int64_t i = 0; i < n; ++i) {
    Rec& r = initial[i];
    memset(&r, 0, sizeof r);
    r.orig_id = (int)i;
    r.strength = v3(1, 1, 1);
    r.start_p = v3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
    r.in_dir = v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
  }
  std::fill(accum, accum + 3 * n, 0.f);
  if (accum2) std::fill(accum2, accum2 + 3 * n, 0.f);
  std::atomic<int64_t> queries(n), shades(0), overflows(0);
  const V3 bgv = v3(bg[0], bg[1], bg[2]);
  // Primary pass with sample_n = sample (trace_runner.cpp:192-213).
  std::vector<IsectResult> prim(n);
  pfor(n, threads, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      prim[i] = kdtree_intersect(*s, initial[i].start_p, initial[i].in_dir);
      if (prim[i].overflow) overflows++;
    }
  });
  std::vector<int> s1_cache;
  for (int64_t i = 0; i < n; ++i) {
    if (prim[i].tri >= 0) {
      initial[i].tri = prim[i].tri;
      initial[i].t = prim[i].t;
      s1_cache.push_back((int)i);
    } else {
      V3 val = (float)sample * (bgv * initial[i].strength);
      accum[3 * i] = val.x; accum[3 * i + 1] = val.y; accum[3 * i + 2] = val.z;
      if (accum2) {
        V3 one = bgv * initial[i].strength;
        accum2[3 * i] = (float)sample * one.x * one.x;
        accum2[3 * i + 1] = (float)sample * one.y * one.y;
        accum2[3 * i + 2] = (float)sample * one.z * one.z;
      }
    }
  }
  // Per-lane seeds (trace_runner.cpp:175-178), from a seeded generator.
  std::vector<int64_t> v_seed(n);
  std::mt19937 gen((uint32_t)seed);
  for (int64_t i = 0; i < n; ++i) v_seed[i] = (int64_t)(gen() & 0x7FFFFFFF);
  std::vector<float> sample_acc(3 * n);
  std::vector<Rec> data;
  std::vector<int> S0, S1, S2[4];
  std::vector<V3> contrib;
  std::vector<int> br, alive;
  for (int ii = 0; ii < sample; ++ii) {
    data = initial;
    S1 = s1_cache;
    S0.clear();
    std::fill(sample_acc.begin(), sample_acc.end(), 0.f);
    for (int i = 0; i < depth; ++i) {
      if (!S0.empty()) {  // kdtree_intersect with sample_n = 1
        std::vector<IsectResult> res(S0.size());
        pfor((int64_t)S0.size(), threads, [&](int64_t b, int64_t e) {
          for (int64_t k = b; k < e; ++k) {
            Rec& r = data[S0[k]];
            res[k] = kdtree_intersect(*s, r.start_p, r.in_dir);
            if (res[k].overflow) overflows++;
          }
        });
        queries += (int64_t)S0.size();
        S1.clear();
        for (size_t k = 0; k < S0.size(); ++k) {
          Rec& r = data[S0[k]];
          if (res[k].tri >= 0) {
            r.tri = res[k].tri;
            r.t = res[k].t;
            S1.push_back(S0[k]);
          } else {
            V3 val = 1.0f * (bgv * r.strength);
            float* a = &sample_acc[3 * r.orig_id];
            a[0] += val.x; a[1] += val.y; a[2] += val.z;
          }
        }
        S0.clear();
      }
      // s1_run over S1 (global_id = position in S1)
      contrib.assign(S1.size(), V3{0, 0, 0});
      br.assign(S1.size(), -1);
      pfor((int64_t)S1.size(), threads, [&](int64_t b, int64_t e) {
        for (int64_t k = b; k < e; ++k) {
          Rec& r = data[S1[k]];
          int64_t sd;
          if (rng_mode == 0) {
            sd = v_seed[k] + k;
          } else {
            sd = (int64_t)path_seed(seed, (uint32_t)r.orig_id, (uint32_t)ii, (uint32_t)i);
          }
          br[k] = s1_run(*s, r, disable_diffuse, &sd, &contrib[k]);
          if (rng_mode == 0) {
            if (br[k] >= 0) v_seed[k] = sd;  // written back after the draw only
          } else {
            v_seed[S1[k]] = sd;  // the path's stream continues in s2
          }
        }
      });
      shades += (int64_t)S1.size();
      for (int k = 0; k < 4; ++k) S2[k].clear();
      for (size_t k = 0; k < S1.size(); ++k) {
        const Rec& r = data[S1[k]];
        float* a = &sample_acc[3 * r.orig_id];
        a[0] += contrib[k].x; a[1] += contrib[k].y; a[2] += contrib[k].z;
        if (br[k] >= 0) S2[br[k]].push_back(S1[k]);
      }
      S1.clear();
      if (i == depth - 1) break;
      // s2 kernels in launch order: refract, specular, diffuse, light
      for (int b = 0; b < 4; ++b) {
        const std::vector<int>& L = S2[b];
        alive.assign(L.size(), 0);
        pfor((int64_t)L.size(), threads, [&](int64_t lo, int64_t hi) {
          for (int64_t k = lo; k < hi; ++k) {
            Rec& r = data[L[k]];
            if (rng_mode == 0) {
              int64_t sd = v_seed[k] + k;
              alive[k] = s2_run(*s, b, r, &sd);
              // s2_refract_run draws nothing; s2_light_run returns before
              // touching v_seed when there are no lights (kernel.cl:522).
              if (b == 1 || b == 2 || (b == 3 && s->num_lights > 0)) v_seed[k] = sd;
            } else {
              int64_t sd = v_seed[L[k]];
              alive[k] = s2_run(*s, b, r, &sd);
            }
          }
        });
        for (size_t k = 0; k < L.size(); ++k)
          if (alive[k]) S0.push_back(L[k]);
      }
    }
    for (int64_t r = 0; r < n; ++r) {
      if (prim[r].tri < 0) continue;
      for (int c = 0; c < 3; ++c) {
        float x = sample_acc[3 * r + c];
        accum[3 * r + c] += x;
        if (accum2) accum2[3 * r + c] += x * x;
      }
    }
  }
  if (counts) {
    counts[0] = queries;
    counts[1] = shades;
    counts[2] = overflows;
  }
}

}  // extern "C"
