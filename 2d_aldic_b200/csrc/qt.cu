// qt.cu -- quadtree meshes: GenerateQuadtreeMesh.m on the host, and the
// device operators of Subpb2Quadtree.m, funGlobalNodalStrainQuadtree.m and
// the refill of flagged nodes on such a mesh.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include <mutex>

#include "qt.cuh"

namespace {
// Device slabs of released meshes, kept for the next mesh of the same device:
// a quadtree frame replaces its mesh on every search frame, and a free plus a
// fresh allocation of the slab each time would put cudaFree's device
// synchronisation and the allocator's page mapping on the frame's path.
struct SlabCache {
  std::mutex mu;
  struct Entry {
    int device;
    aldic::DevBuf buf;
  };
  std::vector<Entry> free;
  static constexpr size_t kMax = 4;
};
SlabCache &slab_cache() {
  static SlabCache c;
  return c;
}
}  // namespace

void aldic_qt_mesh::release() {
  aldic::DevBuf *b[] = {&d_coords, &d_elems, &d_row, &d_col, &d_dpos, &d_iptr, &d_inc, &d_ipos,
                        &d_kind, &d_val, &d_diag, &d_ke, &d_be, &d_es, &d_arow, &d_acol,
                        &d_aval, &d_adiag, &d_valM, &d_diagM};
  for (auto *x : b) {  // views into the slab
    x->p = nullptr;
    x->cap = 0;
  }
  if (slab.p && device >= 0) {
    SlabCache &c = slab_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.free.size() < SlabCache::kMax) {
      c.free.push_back({device, slab});
      slab.p = nullptr;
      slab.cap = 0;
    }
  }
  slab.release();
  device = -1;
}

// a cached slab of this device with at least `bytes`, the smallest that fits
static void take_cached_slab(aldic::DevBuf &slab, int dev, size_t bytes) {
  SlabCache &c = slab_cache();
  std::lock_guard<std::mutex> lk(c.mu);
  int best = -1;
  for (size_t k = 0; k < c.free.size(); ++k)
    if (c.free[k].device == dev && c.free[k].buf.cap >= bytes &&
        (best < 0 || c.free[k].buf.cap < c.free[(size_t)best].buf.cap))
      best = (int)k;
  if (best < 0) return;
  slab.release();
  slab = c.free[(size_t)best].buf;
  c.free.erase(c.free.begin() + best);
}

namespace aldic {

namespace {

// ------------------------------------------------------------------ host mesh
struct HMesh {
  std::vector<double> x, y;                  // node coordinates (0-based index)
  std::vector<std::array<int, 4>> el;        // 1-based corners
  std::vector<std::array<int, 3>> irr;       // sorted parent edge, hanging node
};

// element bounding box in whole pixels; false if not whole or out of the mask
bool box(const HMesh &m, const std::array<int, 4> &e, int W, int H, int b[4]) {
  double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
  for (int c = 0; c < 4; ++c) {
    const double x = m.x[e[c] - 1], y = m.y[e[c] - 1];
    x0 = std::min(x0, x); x1 = std::max(x1, x);
    y0 = std::min(y0, y); y1 = std::max(y1, y);
  }
  if (x0 != std::floor(x0) || x1 != std::floor(x1) || y0 != std::floor(y0) || y1 != std::floor(y1))
    return false;
  b[0] = (int)x0; b[1] = (int)x1; b[2] = (int)y0; b[3] = (int)y1;
  return b[0] >= 1 && b[1] <= W && b[2] >= 1 && b[3] <= H;
}

// Mask box queries.  A mask of zeros and ones (the usual ImgRefMask) is
// answered exactly from a summed-area table of pixel counts: a box straddles
// the edge iff 0 < count < area, and its sum is the count.  Other masks scan
// the box.
struct MaskTable {
  std::vector<int32_t> sat;  // (W+1) x (H+1) counts of ones
  int W = 0, H = 0;
  uint64_t hash = 0;         // of the mask it was built from
  bool binary = false;
};

// FNV-1a over the words of m[0, n) in 8 interleaved lanes (independent
// multiply chains), the lanes folded by one more FNV round each
uint64_t fnv8(const double *m, long long n) {
  uint64_t lane[8];
  for (int j = 0; j < 8; ++j) lane[j] = 1469598103934665603ull + (uint64_t)j;
  long long k = 0;
  for (; k + 8 <= n; k += 8) {
    uint64_t bits[8];
    std::memcpy(bits, m + k, 64);
    for (int j = 0; j < 8; ++j) lane[j] = (lane[j] ^ bits[j]) * 1099511628211ull;
  }
  for (; k < n; ++k) {
    uint64_t bits;
    std::memcpy(&bits, m + k, 8);
    lane[0] = (lane[0] ^ bits) * 1099511628211ull;
  }
  uint64_t h = 1469598103934665603ull;
  for (int j = 0; j < 8; ++j) h = (h ^ lane[j]) * 1099511628211ull;
  return h;
}

// Hash of a whole mask: fixed chunks hashed on up to 8 host threads (the
// scan is bound by one core's memory bandwidth), folded in chunk order, so
// the value does not depend on the thread count.
uint64_t mask_hash(const double *m, long long n) {
  constexpr int kChunks = 8;
  uint64_t part[kChunks];
  const long long per = (n + kChunks - 1) / kChunks;
  auto run = [&](int c) {
    const long long a = std::min(n, c * per), b = std::min(n, a + per);
    part[c] = fnv8(m + a, b - a);
  };
  const unsigned hw = std::thread::hardware_concurrency();
  if (n < (1LL << 20) || hw < 2) {
    for (int c = 0; c < kChunks; ++c) run(c);
  } else {
    std::vector<std::thread> th;
    for (int c = 1; c < kChunks; ++c) th.emplace_back(run, c);
    run(0);
    for (auto &t : th) t.join();
  }
  uint64_t h = 1469598103934665603ull;
  for (int c = 0; c < kChunks; ++c) h = (h ^ part[c]) * 1099511628211ull;
  return h;
}

struct MaskQ {
  const double *mask;
  int W, H;
  bool binary;
  std::vector<int32_t> &sat;
  static MaskTable &table() {
    // kept across calls: a quadtree frame regenerates its mesh on every
    // search frame of a sequence, with the same mask
    static thread_local MaskTable t;
    return t;
  }
  MaskQ(const double *m, int w, int h) : mask(m), W(w), H(h), binary(true), sat(table().sat) {
    MaskTable &t = table();
    const long long n = (long long)W * H;
    const uint64_t hs = mask_hash(m, n);
    if (t.W == W && t.H == H && t.hash == hs && !t.sat.empty()) {
      binary = t.binary;
      return;
    }
    for (long long k = 0; k < n && binary; ++k) binary = m[k] == 0.0 || m[k] == 1.0;
    t.W = W;
    t.H = H;
    t.hash = hs;
    t.binary = binary;
    if (!binary) {
      t.sat.clear();
      t.W = 0;
      return;
    }
    const size_t W1 = (size_t)W + 1;
    if (sat.size() < W1 * (H + 1)) sat.resize(W1 * (H + 1));
    for (size_t x = 0; x < W1; ++x) sat[x] = 0;
    for (int y = 1; y <= H; ++y) {
      int32_t row = 0;
      sat[(size_t)y * W1] = 0;
      for (int x = 1; x <= W; ++x) {
        row += m[(long long)(y - 1) * W + (x - 1)] != 0.0;
        sat[(size_t)y * W1 + x] = sat[(size_t)(y - 1) * W1 + x] + row;
      }
    }
  }
  int64_t count(const int b[4]) const {  // ones in [b0, b1] x [b2, b3], 1-based inclusive
    const size_t W1 = W + 1;
    return sat[(size_t)b[3] * W1 + b[1]] - sat[(size_t)(b[2] - 1) * W1 + b[1]] -
           sat[(size_t)b[3] * W1 + (b[0] - 1)] + sat[(size_t)(b[2] - 1) * W1 + (b[0] - 1)];
  }
  bool straddles(const int b[4]) const {
    if (binary) {
      const int64_t c = count(b), area = (int64_t)(b[1] - b[0] + 1) * (b[3] - b[2] + 1);
      return c > 0 && c < area;
    }
    double lo = 1e300, hi = -1e300;
    for (int y = b[2]; y <= b[3]; ++y)
      for (int x = b[0]; x <= b[1]; ++x) {
        const double v = mask[(long long)(y - 1) * W + (x - 1)];
        lo = std::min(lo, v);
        hi = std::max(hi, v);
      }
    return hi - lo > 0;
  }
  double sum(const int b[4]) const {
    if (binary) return (double)count(b);
    double s = 0;
    for (int y = b[2]; y <= b[3]; ++y)
      for (int x = b[0]; x <= b[1]; ++x) s += mask[(long long)(y - 1) * W + (x - 1)];
    return s;
  }
};

// funMarkEdge.m: box straddles the mask edge and its smaller side > min_size
int mark_edge(const HMesh &m, const MaskQ &mq, double min_size, std::vector<int> &out) {
  out.clear();
  for (size_t e = 0; e < m.el.size(); ++e) {
    int b[4];
    if (!box(m, m.el[e], mq.W, mq.H, b)) return E_ARG;
    const double size = std::min(std::abs(b[1] - b[0]), std::abs(b[3] - b[2]));
    if (size > min_size && mq.straddles(b)) out.push_back((int)e);
  }
  return OK;
}

// Sort (edge key, occurrence) pairs by key, ties in occurrence order: the
// pairs arrive in occurrence order, so a stable LSD radix sort on the two
// node numbers (each below nn + 1) gives the order of sorting the pairs.
void sort_edges(std::vector<std::pair<uint64_t, int>> &ed, size_t nn) {
  int bits = 1;
  while (((size_t)1 << bits) <= nn + 1) ++bits;
  const int digit = 11, R = 1 << digit;
  std::vector<std::pair<uint64_t, int>> tmp(ed.size());
  std::vector<size_t> cnt(R);
  // low node (bits 0..31) then high node (bits 32..63), digit by digit
  for (int half = 0; half < 2; ++half)
    for (int lo = 0; lo < bits; lo += digit) {
      const int sh = 32 * half + lo;
      std::fill(cnt.begin(), cnt.end(), 0);
      for (const auto &v : ed) ++cnt[(v.first >> sh) & (R - 1)];
      size_t sum = 0;
      for (int d = 0; d < R; ++d) {
        const size_t c = cnt[d];
        cnt[d] = sum;
        sum += c;
      }
      for (const auto &v : ed) tmp[cnt[(v.first >> sh) & (R - 1)]++] = v;
      ed.swap(tmp);
    }
}

// provideGeometricData.m: edges of the irregular triples (column by column)
// then of the elements, sorted unique; inverse maps per triple / element
struct Geo {
  std::vector<std::array<int, 2>> e2n;
  std::vector<std::array<int, 3>> irr2e;
  std::vector<std::array<int, 4>> el2e;
};

void geometric(const HMesh &m, Geo &g) {
  const size_t ni = m.irr.size(), ne = m.el.size(), n3 = 3 * ni;
  // (sorted node pair as one 64-bit key, occurrence index), sorted
  std::vector<std::pair<uint64_t, int>> ed;
  ed.reserve(n3 + 4 * ne);
  auto k2 = [](int a, int b) {
    return ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint64_t)(uint32_t)std::max(a, b);
  };
  for (int c = 0; c < 3; ++c)
    for (size_t r = 0; r < ni; ++r)
      ed.push_back({k2(m.irr[r][c], m.irr[r][(c + 1) % 3]), (int)(c * ni + r)});
  for (int c = 0; c < 4; ++c)
    for (size_t r = 0; r < ne; ++r)
      ed.push_back({k2(m.el[r][c], m.el[r][(c + 1) % 4]), (int)(n3 + c * ne + r)});
  sort_edges(ed, m.x.size());
  std::vector<int> ie(ed.size());
  g.e2n.clear();
  for (size_t k = 0; k < ed.size(); ++k) {
    if (k == 0 || ed[k].first != ed[k - 1].first)
      g.e2n.push_back({(int)(ed[k].first >> 32), (int)(ed[k].first & 0xffffffffu)});
    ie[ed[k].second] = (int)g.e2n.size() - 1;
  }
  g.irr2e.assign(ni, {0, 0, 0});
  g.el2e.assign(ne, {0, 0, 0, 0});
  for (int c = 0; c < 3; ++c)
    for (size_t r = 0; r < ni; ++r) g.irr2e[r][c] = ie[c * ni + r];
  for (int c = 0; c < 4; ++c)
    for (size_t r = 0; r < ne; ++r) g.el2e[r][c] = ie[n3 + c * ne + r];
}

// QrefineR.m: red refinement of the marked elements, closure by the
// 1-irregular rule, new nodes on edges (sorted edge order) then at the
// centres of refined elements (element order)
void qrefine(HMesh &m, const std::vector<int> &marked) {
  Geo g;
  geometric(m, g);
  const size_t nE = m.el.size(), ni = m.irr.size();
  std::vector<long long> e2n(g.e2n.size(), 0);
  for (int e : marked)
    for (int c = 0; c < 4; ++c) e2n[g.el2e[e][c]] = 1;
  for (size_t r = 0; r < ni; ++r) e2n[g.irr2e[r][0]] = 1;
  bool first = true;
  size_t nk = 0, nswap = 0;
  std::vector<int> kdx;
  while (first || nk || nswap) {
    first = false;
    kdx.clear();
    for (size_t e = 0; e < nE; ++e) {
      long long s = 0, mn = 1;
      for (int c = 0; c < 4; ++c) {
        const long long v = e2n[g.el2e[e][c]];
        s += v < 0 ? -v : v;
        mn = std::min(mn, v);
      }
      if (s < 4 && (s > 2 || mn < 0)) kdx.push_back((int)e);
    }
    for (int e : kdx)
      for (int c = 0; c < 4; ++c)
        if (e2n[g.el2e[e][c]] == 0) e2n[g.el2e[e][c]] = 1;
    nk = kdx.size();
    nswap = 0;
    if (ni) {
      std::vector<int> sw;
      for (size_t r = 0; r < ni; ++r)
        if (e2n[g.irr2e[r][1]] != 0 || e2n[g.irr2e[r][2]] != 0)
          if (e2n[g.irr2e[r][0]] != -1) sw.push_back(g.irr2e[r][0]);
      for (int ed : sw) e2n[ed] = -1;
      nswap = sw.size();
    }
  }
  for (size_t r = 0; r < ni; ++r) e2n[g.irr2e[r][0]] = -1;
  long long next = (long long)m.x.size() + 1;
  for (size_t ed = 0; ed < e2n.size(); ++ed)
    if (e2n[ed] > 0) {
      e2n[ed] = next++;
      const int a = g.e2n[ed][0] - 1, b = g.e2n[ed][1] - 1;
      m.x.push_back((m.x[a] + m.x[b]) / 2);
      m.y.push_back((m.y[a] + m.y[b]) / 2);
    }
  for (size_t r = 0; r < ni; ++r) e2n[g.irr2e[r][0]] = m.irr[r][2];
  std::vector<std::array<long long, 4>> nn(nE);
  std::vector<int> reftyp(nE);
  for (size_t e = 0; e < nE; ++e) {
    int t = 0;
    for (int c = 0; c < 4; ++c) {
      nn[e][c] = e2n[g.el2e[e][c]];
      if (nn[e][c] != 0) t |= 1 << c;
    }
    reftyp[e] = t;
  }
  std::vector<long long> mid(nE, 0);
  for (size_t e = 0; e < nE; ++e)
    if (reftyp[e] == 15) {
      mid[e] = (long long)m.x.size() + 1;
      const auto &q = m.el[e];
      m.x.push_back((m.x[q[0] - 1] + m.x[q[1] - 1] + m.x[q[2] - 1] + m.x[q[3] - 1]) / 4);
      m.y.push_back((m.y[q[0] - 1] + m.y[q[1] - 1] + m.y[q[2] - 1] + m.y[q[3] - 1]) / 4);
    }
  std::vector<std::array<int, 4>> nel;
  nel.reserve(nE * 2);
  for (size_t e = 0; e < nE; ++e) {
    const auto &q = m.el[e];
    if (reftyp[e] < 15) {
      nel.push_back(q);
    } else {
      const int md = (int)mid[e];
      const auto &w = nn[e];
      nel.push_back({q[0], (int)w[0], md, (int)w[3]});
      nel.push_back({q[1], (int)w[1], md, (int)w[0]});
      nel.push_back({q[2], (int)w[2], md, (int)w[1]});
      nel.push_back({q[3], (int)w[3], md, (int)w[2]});
    }
  }
  // new irregularity data, in the column-major order of MATLAB's find()
  std::vector<std::array<int, 3>> nirr;
  for (int c = 0; c < 4; ++c)
    for (size_t e = 0; e < nE; ++e)
      if (reftyp[e] > 0 && reftyp[e] < 15 && nn[e][c] != 0) {
        const auto &p = g.e2n[g.el2e[e][c]];
        nirr.push_back({p[0], p[1], (int)nn[e][c]});
      }
  for (int c = 0; c < 2; ++c)
    for (size_t r = 0; r < ni; ++r) {
      const long long v1 = e2n[g.irr2e[r][1]], v2 = e2n[g.irr2e[r][2]];
      if (v1 + v2 == 0) continue;
      const long long v = c == 0 ? v1 : v2;
      if (v != 0) {
        const auto &p = g.e2n[g.irr2e[r][1 + c]];
        nirr.push_back({p[0], p[1], (int)v});
      }
    }
  m.el.swap(nel);
  m.irr.swap(nirr);
}

}  // namespace

// Open-addressing table of nonzero 64-bit keys -> int (initially -1), for the
// hanging-node lookups of qt_generate (a few thousand keys, ~10^5 probes).
struct FlatMap {
  std::vector<uint64_t> k;
  std::vector<int> v;
  size_t mask;
  explicit FlatMap(size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    k.assign(cap, 0);
    v.assign(cap, -1);
    mask = cap - 1;
  }
  static size_t mix(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    return (size_t)x;
  }
  void insert(uint64_t key) {
    for (size_t i = mix(key) & mask;; i = (i + 1) & mask) {
      if (k[i] == key) return;
      if (k[i] == 0) {
        k[i] = key;
        return;
      }
    }
  }
  int *find(uint64_t key) {
    for (size_t i = mix(key) & mask;; i = (i + 1) & mask) {
      if (k[i] == key) return &v[i];
      if (k[i] == 0) return nullptr;
    }
  }
};

int qt_generate(int n0, const double *coords, int ne0, const int32_t *elems, const double *mask,
                int W, int H, double step, int min_size, aldic_qt_mesh &out) {
  ALDIC_CHECK(n0 >= 4 && ne0 >= 1 && coords && elems && mask && W > 0 && H > 0 && step > 0 &&
                  min_size >= 1,
              E_ARG, "qt_mesh_generate: bad arguments");
  HMesh m;
  m.x.assign(coords, coords + n0);
  m.y.assign(coords + n0, coords + 2 * n0);
  m.el.resize(ne0);
  for (int e = 0; e < ne0; ++e)
    for (int c = 0; c < 4; ++c) {
      const int v = elems[(long long)c * ne0 + e];
      ALDIC_CHECK(v >= 1 && v <= n0, E_ARG, "qt_mesh_generate: element node out of range");
      m.el[e][c] = v;
    }
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
  for (int k = 0; k < n0; ++k) {
    xmin = std::min(xmin, m.x[k]); xmax = std::max(xmax, m.x[k]);
    ymin = std::min(ymin, m.y[k]); ymax = std::max(ymax, m.y[k]);
  }
  const MaskQ mq(mask, W, H);
  std::vector<int> mk;
  for (int pass = 0;; ++pass) {
    ALDIC_CHECK(pass < 64, E_ARG, "qt_mesh_generate: refinement does not terminate");
    if (mark_edge(m, mq, 2.0 * min_size, mk) != OK) {
      set_error("qt_mesh_generate: element corners must be whole pixels inside the mask "
                "(uniform step a power-of-two multiple of the minimum element size)");
      return E_ARG;
    }
    qrefine(m, mk);
    if (mk.empty()) break;
  }
  // hanging nodes into slots 5-8 (GenerateQuadtreeMesh.m:40-57): the first
  // element whose edge (c1, c2), in either direction, is the parent edge
  const size_t ne = m.el.size();
  std::vector<std::array<int, 8>> E(ne);
  for (size_t e = 0; e < ne; ++e) {
    for (int c = 0; c < 4; ++c) E[e][c] = m.el[e][c];
    for (int c = 4; c < 8; ++c) E[e][c] = 0;
  }
  static const int pairs[8][3] = {{0, 1, 7}, {1, 2, 4}, {2, 3, 5}, {3, 0, 6},
                                  {1, 0, 7}, {2, 1, 4}, {3, 2, 5}, {0, 3, 6}};
  // (corner a, corner b, pair) -> first element: only the pairs that are
  // parent edges of hanging nodes are looked up, so only those are recorded
  auto key = [](int a, int b, int pi) -> unsigned long long {
    return ((unsigned long long)(unsigned)a << 35) ^ ((unsigned long long)(unsigned)b << 3) ^
           (unsigned long long)pi;
  };
  FlatMap first(8 * m.irr.size());
  for (const auto &r : m.irr)
    for (int pi = 0; pi < 8; ++pi) first.insert(key(r[0], r[1], pi));
  for (int pi = 0; pi < 8; ++pi)
    for (size_t e = 0; e < ne; ++e) {
      int *v = first.find(key(m.el[e][pairs[pi][0]], m.el[e][pairs[pi][1]], pi));
      if (v && *v < 0) *v = (int)e;
    }
  for (const auto &r : m.irr)
    for (int pi = 0; pi < 8; ++pi) {
      const int e = *first.find(key(r[0], r[1], pi));
      if (e >= 0) E[e][pairs[pi][2]] = r[2];
    }
  // funMarkInside.m: drop elements less than half inside the mask
  std::vector<std::array<int, 8>> K;
  for (size_t e = 0; e < ne; ++e) {
    int b[4];
    if (!box(m, m.el[e], W, H, b)) return E_ARG;
    const double s = mq.sum(b);
    if (!(s < 0.5 * (b[1] - b[0]) * (b[3] - b[2]))) K.push_back(E[e]);
  }
  // Dirichlet nodes (GenerateQuadtreeMesh.m:75-110): refined elements and
  // elements at the ROI border, grown by two rings of neighbours
  const size_t nk = K.size();
  std::vector<char> sel(nk, 0);
  for (size_t e = 0; e < nk; ++e) {
    const int a = K[e][0] - 1, c = K[e][2] - 1;
    const double d = std::hypot(m.x[a] - m.x[c], m.y[a] - m.y[c]);
    sel[e] = d < 0.99 * std::sqrt(2.0) * step || m.x[a] < xmin + 1.01 * step ||
             m.x[c] > xmax - 1.01 * step || m.y[a] < ymin + 1.01 * step ||
             m.y[c] > ymax - 1.01 * step;
  }
  const size_t nn = m.x.size();
  std::vector<char> mark(nn + 1, 0);
  for (size_t e = 0; e < nk; ++e)
    if (sel[e])
      for (int s = 0; s < 8; ++s) mark[K[e][s]] = 1;
  mark[0] = 0;
  for (int it = 0; it < 2; ++it) {
    std::vector<char> nm(nn + 1, 0);
    for (size_t e = 0; e < nk; ++e) {
      bool hit = false;
      for (int s = 0; s < 8; ++s)
        if (K[e][s] && mark[K[e][s]]) hit = true;
      if (hit)
        for (int s = 0; s < 8; ++s) nm[K[e][s]] = 1;
    }
    nm[0] = 0;
    mark.swap(nm);
  }
  out.release();
  out.n = (int)nn;
  out.ne = (int)nk;
  out.coords.resize(2 * nn);
  for (size_t k = 0; k < nn; ++k) {
    out.coords[k] = m.x[k];
    out.coords[nn + k] = m.y[k];
  }
  out.elems.resize(8 * nk);
  for (size_t e = 0; e < nk; ++e)
    for (int s = 0; s < 8; ++s) out.elems[(size_t)s * nk + e] = K[e][s];
  out.dirichlet.clear();
  for (size_t k = 1; k <= nn; ++k)
    if (mark[k]) out.dirichlet.push_back((int)k);
  return OK;
}

// ------------------------------------------------------------------ device
namespace {

constexpr double kG = 0.57735026918962576451;  // 1/sqrt(3)

__device__ __forceinline__ double sgn(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); }

// N1..N8 and d/dksi, d/deta with hanging-node enrichment (Subpb2Quadtree.m
// shape functions and the funDN* helpers); d[4] = presence of slots 5-8
__device__ __forceinline__ void shape8(double ksi, double eta, const double d[4], double N[8],
                                       double dk[8], double de[8]) {
  const double ak = fabs(ksi), ae = fabs(eta);
  N[4] = d[0] * 0.5 * (1 + ksi) * (1 - ae);
  N[5] = d[1] * 0.5 * (1 + eta) * (1 - ak);
  N[6] = d[2] * 0.5 * (1 - ksi) * (1 - ae);
  N[7] = d[3] * 0.5 * (1 - eta) * (1 - ak);
  N[0] = (1 - ksi) * (1 - eta) * 0.25 - 0.5 * (N[6] + N[7]);
  N[1] = (1 + ksi) * (1 - eta) * 0.25 - 0.5 * (N[7] + N[4]);
  N[2] = (1 + ksi) * (1 + eta) * 0.25 - 0.5 * (N[4] + N[5]);
  N[3] = (1 - ksi) * (1 + eta) * 0.25 - 0.5 * (N[5] + N[6]);
  dk[4] = d[0] * 0.5 * (1 - ae);
  de[4] = d[0] * 0.5 * (1 + ksi) * sgn(-eta);
  dk[5] = d[1] * 0.5 * (1 + eta) * sgn(-ksi);
  de[5] = d[1] * 0.5 * (1 - ak);
  dk[6] = d[2] * 0.5 * (-1) * (1 - ae);
  de[6] = d[2] * 0.5 * (1 - ksi) * sgn(-eta);
  dk[7] = d[3] * 0.5 * (1 - eta) * sgn(-ksi);
  de[7] = d[3] * 0.5 * (-1) * (1 - ak);
  dk[0] = -0.25 * (1 - eta) - 0.5 * (dk[6] + dk[7]);
  de[0] = -0.25 * (1 - ksi) - 0.5 * (de[6] + de[7]);
  dk[1] = 0.25 * (1 - eta) - 0.5 * (dk[7] + dk[4]);
  de[1] = -0.25 * (1 + ksi) - 0.5 * (de[7] + de[4]);
  dk[2] = 0.25 * (1 + eta) - 0.5 * (dk[4] + dk[5]);
  de[2] = 0.25 * (1 + ksi) - 0.5 * (de[4] + de[5]);
  dk[3] = -0.25 * (1 + eta) - 0.5 * (dk[5] + dk[6]);
  de[3] = 0.25 * (1 - ksi) - 0.5 * (de[5] + de[6]);
}

// d/dx, d/dy and det J at (ksi, eta)
__device__ __forceinline__ double grads(const double dk[8], const double de[8], const double px[8],
                                        const double py[8], double dx[8], double dy[8]) {
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    J11 += dk[s] * px[s];
    J12 += dk[s] * py[s];
    J21 += de[s] * px[s];
    J22 += de[s] * py[s];
  }
  const double det = J11 * J22 - J12 * J21;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    dx[s] = (J22 * dk[s] - J12 * de[s]) / det;
    dy[s] = (-J21 * dk[s] + J11 * de[s]) / det;
  }
  return det;
}

// one thread per (element, local row a): row a of the scalar 8x8 element
// matrix sum_gp detJ (beta grad Na . grad Nb + mu Na Nb) and the row's
// right-hand sides (the duals are multiplied by zero in the reference)
__global__ void k_qt_elem(int ne, const int *__restrict__ E, const double *__restrict__ cx,
                          const double *__restrict__ cy, double beta, double mu,
                          const double *__restrict__ U, const double *__restrict__ F,
                          double *__restrict__ ke, double *__restrict__ be) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 8LL * ne) return;
  const int e = (int)(t >> 3), a = (int)(t & 7);
  int nd[8];
  double px[8], py[8], d[4];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    nd[s] = E[e * 8 + s];
    px[s] = nd[s] >= 0 ? cx[nd[s]] : 0.0;
    py[s] = nd[s] >= 0 ? cy[nd[s]] : 0.0;
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) d[s] = nd[4 + s] >= 0 ? 1.0 : 0.0;
  double K[8] = {0, 0, 0, 0, 0, 0, 0, 0}, bu = 0, bv = 0;
  if (nd[a] >= 0) {
    const int ka = nd[a];
    const double F0 = F[4 * ka], F1 = F[4 * ka + 1], F2 = F[4 * ka + 2], F3 = F[4 * ka + 3];
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
      const double ksi = (g & 1) ? kG : -kG, eta = (g & 2) ? kG : -kG;
      double N[8], dk[8], de[8], dx[8], dy[8];
      shape8(ksi, eta, d, N, dk, de);
      const double J = grads(dk, de, px, py, dx, dy);
      double uu = 0, vv = 0;
#pragma unroll
      for (int s = 0; s < 8; ++s)
        if (nd[s] >= 0) {
          uu += N[s] * U[2 * nd[s]];
          vv += N[s] * U[2 * nd[s] + 1];
        }
#pragma unroll
      for (int s = 0; s < 8; ++s)
        if (nd[s] >= 0) K[s] += J * (beta * (dx[a] * dx[s] + dy[a] * dy[s]) + mu * N[a] * N[s]);
      bu += J * (beta * (dx[a] * F0 + dy[a] * F2) + mu * N[a] * uu);
      bv += J * (beta * (dx[a] * F1 + dy[a] * F3) + mu * N[a] * vv);
    }
  }
#pragma unroll
  for (int s = 0; s < 8; ++s) ke[(long long)e * 64 + a * 8 + s] = K[s];
  be[(long long)e * 16 + a] = bu;
  be[(long long)e * 16 + 8 + a] = bv;
}

// one thread per node: its matrix row and right-hand sides, summed over the
// incident elements in element order (deterministic)
__global__ void k_qt_gather(int n, const int *__restrict__ iptr, const int *__restrict__ inc,
                            const int *__restrict__ ipos, const int *__restrict__ row,
                            const double *__restrict__ ke, const double *__restrict__ be,
                            double *__restrict__ val, double *__restrict__ b) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  for (int p = row[a]; p < row[a + 1]; ++p) val[p] = 0.0;
  double bu = 0, bv = 0;
  for (int t = iptr[a]; t < iptr[a + 1]; ++t) {
    const int ent = inc[t], e = ent >> 3, sa = ent & 7;
    for (int sb = 0; sb < 8; ++sb) {
      const int pos = ipos[8 * t + sb];
      if (pos >= 0) val[pos] += ke[(long long)e * 64 + sa * 8 + sb];
    }
    bu += be[(long long)e * 16 + sa];
    bv += be[(long long)e * 16 + 8 + sa];
  }
  b[a] = bu;
  b[n + a] = bv;
}

// Dirichlet elimination: free rows move the fixed columns to the right-hand
// side (start from U); Dirichlet rows keep U; nodes in no element get 0
__global__ void k_qt_elim(int n, const int *__restrict__ row, const int *__restrict__ col,
                          const double *__restrict__ val, const int *__restrict__ dpos,
                          const unsigned char *__restrict__ kind, const double *__restrict__ U,
                          double *__restrict__ b, double *__restrict__ x,
                          unsigned char *__restrict__ mask, double *__restrict__ diag) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int kd = kind[a];
  diag[a] = kd == 2 ? 1.0 : val[dpos[a]];
  for (int f = 0; f < 2; ++f) {
    const long long o = (long long)f * n + a;
    if (kd == 0) {
      double s = b[o];
      for (int p = row[a]; p < row[a + 1]; ++p) {
        const int c = col[p];
        if (kind[c] == 1) s -= val[p] * U[2 * c + f];
      }
      b[o] = s;
      x[o] = U[2 * a + f];
      mask[o] = 1;
    } else {
      const double v = kd == 1 ? U[2 * a + f] : 0.0;
      b[o] = v;
      x[o] = v;
      mask[o] = 0;
    }
  }
}

// The beta sweep's three systems from the stiffness (valK, b fields 0-1)
// and mass (valM, b fields 2-3) parts: for beta[q], fields 2q, 2q + 1 of b,
// x and mask as k_qt_elim sets them for beta[q] K + mu M, and the two
// diagonals (each node reads its own four b entries before writing six).
struct QtBetas {
  double v[3];
};
__global__ void k_qt_elim3(int n, const int *__restrict__ row, const int *__restrict__ col,
                           const double *__restrict__ valK, const double *__restrict__ valM,
                           const int *__restrict__ dpos, const unsigned char *__restrict__ kind,
                           const double *__restrict__ U, QtBetas be, double mu,
                           double *__restrict__ b, double *__restrict__ x,
                           unsigned char *__restrict__ mask, double *__restrict__ diagK,
                           double *__restrict__ diagM) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int kd = kind[a];
  diagK[a] = kd == 2 ? 1.0 : valK[dpos[a]];
  diagM[a] = kd == 2 ? 0.0 : valM[dpos[a]];
  const double bK[2] = {b[a], b[(long long)n + a]};
  const double bM[2] = {b[2LL * n + a], b[3LL * n + a]};
  for (int q = 0; q < 3; ++q)
    for (int f = 0; f < 2; ++f) {
      const long long o = (long long)(2 * q + f) * n + a;
      if (kd == 0) {
        double s = be.v[q] * bK[f] + mu * bM[f];
        for (int p = row[a]; p < row[a + 1]; ++p) {
          const int c = col[p];
          if (kind[c] == 1) s -= (be.v[q] * valK[p] + mu * valM[p]) * U[2 * c + f];
        }
        b[o] = s;
        x[o] = U[2 * a + f];
        mask[o] = 1;
      } else {
        const double v = kd == 1 ? U[2 * a + f] : 0.0;
        b[o] = v;
        x[o] = v;
        mask[o] = 0;
      }
    }
}

__global__ void k_qt_store(int n, const double *__restrict__ x, double *__restrict__ Uhat) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  Uhat[2 * a] = x[a];
  Uhat[2 * a + 1] = x[n + a];
}

// Gauss-point strains of an element's Q4 corners (slots 5-8 ignored, as
// funGlobalNodalStrainQuadtree.m:33 zeroes them), extrapolated to its
// corners: es[e][corner][du/dx du/dy dv/dx dv/dy]
__global__ void k_qt_strain_elem(int ne, const int *__restrict__ E, const double *__restrict__ cx,
                                 const double *__restrict__ cy, const double *__restrict__ U,
                                 double *__restrict__ es) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double px[8], py[8], u[4], v[4];
  const double d[4] = {0, 0, 0, 0};
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int k = E[e * 8 + s];
    px[s] = cx[k];
    py[s] = cy[k];
    u[s] = U[2 * k];
    v[s] = U[2 * k + 1];
    px[4 + s] = py[4 + s] = 0.0;
  }
  double gv[4][4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const double ksi = (g & 1) ? kG : -kG, eta = (g & 2) ? kG : -kG;
    double N[8], dk[8], de[8], dx[8], dy[8];
    shape8(ksi, eta, d, N, dk, de);
    grads(dk, de, px, py, dx, dy);
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      a0 += dx[s] * u[s];
      a1 += dy[s] * u[s];
      a2 += dx[s] * v[s];
      a3 += dy[s] * v[s];
    }
    gv[g][0] = a0; gv[g][1] = a1; gv[g][2] = a2; gv[g][3] = a3;
  }
  const double s3 = 1.7320508075688772935;  // corner / Gauss-point ratio
  const double ck[4] = {-s3, s3, s3, -s3}, ce[4] = {-s3, -s3, s3, s3};
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double k = ck[a], q = ce[a];
    const double w0 = (1 - k) * (1 - q) * 0.25, w1 = (1 + k) * (1 - q) * 0.25,
                 w2 = (1 - k) * (1 + q) * 0.25, w3 = (1 + k) * (1 + q) * 0.25;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      es[(long long)e * 16 + a * 4 + c] = w0 * gv[0][c] + w1 * gv[1][c] + w2 * gv[2][c] + w3 * gv[3][c];
  }
}

__global__ void k_qt_strain_gather(int n, const int *__restrict__ iptr, const int *__restrict__ inc,
                                   const double *__restrict__ es, double *__restrict__ F) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double s[4] = {0, 0, 0, 0};
  int cnt = 0;
  for (int t = iptr[a]; t < iptr[a + 1]; ++t) {
    const int ent = inc[t], e = ent >> 3, sa = ent & 7;
    if (sa >= 4) continue;
    for (int c = 0; c < 4; ++c) s[c] += es[(long long)e * 16 + sa * 4 + c];
    cnt++;
  }
  for (int c = 0; c < 4; ++c) F[4 * a + c] = cnt ? s[c] / cnt : 0.0;
}

// refill: bad nodes are unknowns of (L + t I) x = sum of good neighbours;
// the nf interleaved fields of vals go to solver fields f0 .. f0 + nf - 1
__global__ void k_qt_fill_prep(int n, int nf, int f0, const double *__restrict__ vals,
                               const unsigned char *__restrict__ bad, const int *__restrict__ row,
                               const int *__restrict__ col, double *__restrict__ b,
                               double *__restrict__ x, unsigned char *__restrict__ mask) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  for (int f = 0; f < nf; ++f) {
    const long long o = (long long)(f0 + f) * n + a;
    if (bad[a]) {
      double s = 0.0;
      for (int p = row[a]; p < row[a + 1]; ++p) {
        const int c = col[p];
        if (c != a && !bad[c]) s += vals[(long long)c * nf + f];
      }
      b[o] = s;
      x[o] = 0.0;
      mask[o] = 1;
    } else {
      const double v = vals[(long long)a * nf + f];
      b[o] = v;
      x[o] = v;
      mask[o] = 0;
    }
  }
}

__global__ void k_qt_fill_store(int n, int nf, int f0, const double *__restrict__ x,
                                const unsigned char *__restrict__ bad, double *__restrict__ vals) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n || !bad[a]) return;
  for (int f = 0; f < nf; ++f) vals[(long long)a * nf + f] = x[(long long)(f0 + f) * n + a];
}

inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }


}  // namespace

int qt_upload(aldic_qt_mesh &m, cudaStream_t st) {
  int dev = 0;
  ALDIC_CUDA(cudaGetDevice(&dev));
  if (m.device == dev) return OK;
  m.release();
  const int n = m.n, ne = m.ne;
  std::vector<int> E(8 * (size_t)ne);
  std::vector<unsigned char> kind(n, 2);
  for (int e = 0; e < ne; ++e)
    for (int s = 0; s < 8; ++s) {
      const int v = m.elems[(size_t)s * ne + e];
      ALDIC_CHECK(v >= 0 && v <= n, E_ARG, "quadtree mesh: element node out of range");
      E[8 * e + s] = v - 1;
      if (v) kind[v - 1] = 0;
    }
  ALDIC_CHECK(ne >= 1 && E[0] >= 0, E_ARG, "quadtree mesh: no elements");
  for (int e = 0; e < ne; ++e)
    for (int s = 0; s < 4; ++s) ALDIC_CHECK(E[8 * e + s] >= 0, E_ARG, "quadtree mesh: empty corner slot");
  for (int d : m.dirichlet) {
    ALDIC_CHECK(d >= 1 && d <= n, E_ARG, "quadtree mesh: Dirichlet node out of range");
    if (kind[d - 1] == 0) kind[d - 1] = 1;
  }
  // incidence node -> (element * 8 + slot) in element order (counting sort)
  std::vector<int> iptr(n + 1, 0), inc;
  for (int k = 0; k < 8 * ne; ++k)
    if (E[k] >= 0) iptr[E[k] + 1]++;
  for (int a = 0; a < n; ++a) iptr[a + 1] += iptr[a];
  inc.resize(iptr[n]);
  {
    std::vector<int> fill(iptr.begin(), iptr.end() - 1);
    for (int k = 0; k < 8 * ne; ++k)
      if (E[k] >= 0) inc[fill[E[k]]++] = k;
  }
  // FE pattern: node pairs sharing an element, each row sorted
  std::vector<int> row(n + 1, 0), col, dpos(n, 0), buf;
  col.reserve((size_t)iptr[n] * 4);
  for (int a = 0; a < n; ++a) {
    buf.clear();
    for (int t = iptr[a]; t < iptr[a + 1]; ++t) {
      const int e = inc[t] >> 3;
      for (int b = 0; b < 8; ++b)
        if (E[8 * e + b] >= 0) buf.push_back(E[8 * e + b]);
    }
    std::sort(buf.begin(), buf.end());
    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    row[a + 1] = row[a] + (int)buf.size();
    for (size_t k = 0; k < buf.size(); ++k)
      if (buf[k] == a) dpos[a] = row[a] + (int)k;
    col.insert(col.end(), buf.begin(), buf.end());
  }
  // scatter map of each incidence into its row
  std::vector<int> ipos((size_t)8 * inc.size());
  for (int a = 0; a < n; ++a)
    for (int t = iptr[a]; t < iptr[a + 1]; ++t) {
      const int e = inc[t] >> 3;
      for (int sb = 0; sb < 8; ++sb) {
        const int nb = E[8 * e + sb];
        ipos[(size_t)8 * t + sb] =
            nb < 0 ? -1
                   : (int)(std::lower_bound(col.begin() + row[a], col.begin() + row[a + 1], nb) -
                           col.begin());
      }
    }
  // refill graph: element boundary rings 1-8-2-5-3-6-4-7 (edge list, then
  // grouped per node by a counting sort)
  static const int ring[8] = {0, 7, 1, 4, 2, 5, 3, 6};
  std::vector<int> ea, eb;
  ea.reserve((size_t)16 * ne);
  eb.reserve((size_t)16 * ne);
  for (int e = 0; e < ne; ++e) {
    int r[8], k = 0;
    for (int q = 0; q < 8; ++q)
      if (E[8 * e + ring[q]] >= 0) r[k++] = E[8 * e + ring[q]];
    for (int q = 0; q < k; ++q) {
      const int a = r[q], b = r[(q + 1) % k];
      ea.push_back(a); eb.push_back(b);
      ea.push_back(b); eb.push_back(a);
    }
  }
  std::vector<int> aptr(n + 1, 0), anb(ea.size());
  for (int a : ea) aptr[a + 1]++;
  for (int a = 0; a < n; ++a) aptr[a + 1] += aptr[a];
  {
    std::vector<int> fill(aptr.begin(), aptr.end() - 1);
    for (size_t k = 0; k < ea.size(); ++k) anb[fill[ea[k]]++] = eb[k];
  }
  std::vector<int> arow(n + 1, 0), acol;
  std::vector<double> aval, adiag(n);
  acol.reserve(anb.size() + n);
  aval.reserve(anb.size() + n);
  for (int a = 0; a < n; ++a) {
    auto b0 = anb.begin() + aptr[a], b1 = anb.begin() + aptr[a + 1];
    std::sort(b0, b1);
    b1 = std::unique(b0, b1);
    const double deg = (double)(b1 - b0);
    bool diag_done = false;
    for (auto it = b0; it != b1; ++it) {
      const int v = *it;
      if (!diag_done && v > a) {
        acol.push_back(a);
        aval.push_back(deg + kQtFillTether);
        diag_done = true;
      }
      acol.push_back(v);
      aval.push_back(-1.0);
    }
    if (!diag_done) {
      acol.push_back(a);
      aval.push_back(deg + kQtFillTether);
    }
    adiag[a] = deg + kQtFillTether;
    arow[a + 1] = (int)acol.size();
  }
  // one device slab: the arrays above, then the work arrays
  struct Part {
    DevBuf *b;
    const void *src;
    size_t bytes;
  };
  const Part parts[] = {
      {&m.d_coords, m.coords.data(), sizeof(double) * m.coords.size()},
      {&m.d_elems, E.data(), sizeof(int) * E.size()},
      {&m.d_row, row.data(), sizeof(int) * row.size()},
      {&m.d_col, col.data(), sizeof(int) * col.size()},
      {&m.d_dpos, dpos.data(), sizeof(int) * dpos.size()},
      {&m.d_iptr, iptr.data(), sizeof(int) * iptr.size()},
      {&m.d_inc, inc.data(), sizeof(int) * inc.size()},
      {&m.d_ipos, ipos.data(), sizeof(int) * ipos.size()},
      {&m.d_kind, kind.data(), kind.size()},
      {&m.d_arow, arow.data(), sizeof(int) * arow.size()},
      {&m.d_acol, acol.data(), sizeof(int) * acol.size()},
      {&m.d_aval, aval.data(), sizeof(double) * aval.size()},
      {&m.d_adiag, adiag.data(), sizeof(double) * adiag.size()},
      {&m.d_val, nullptr, sizeof(double) * (col.size() + 1)},
      {&m.d_diag, nullptr, sizeof(double) * n},
      {&m.d_valM, nullptr, sizeof(double) * (col.size() + 1)},
      {&m.d_diagM, nullptr, sizeof(double) * n},
      {&m.d_ke, nullptr, sizeof(double) * 64 * ne},
      {&m.d_be, nullptr, sizeof(double) * 16 * ne},
      {&m.d_es, nullptr, sizeof(double) * 16 * ne},
  };
  size_t off = 0, upload = 0;
  for (const Part &q : parts) {
    off = (off + 255) & ~(size_t)255;
    if (q.src) upload = off + q.bytes;
    off += q.bytes > 0 ? q.bytes : 1;
  }
  int rc;
  take_cached_slab(m.slab, dev, off);
  if ((rc = m.slab.ensure(off))) return rc;
  std::vector<unsigned char> host(upload, 0);
  off = 0;
  for (const Part &q : parts) {
    off = (off + 255) & ~(size_t)255;
    q.b->p = m.slab.as<unsigned char>() + off;
    q.b->cap = 0;  // a view: never grown or freed on its own
    if (q.src && q.bytes) std::memcpy(host.data() + off, q.src, q.bytes);
    off += q.bytes > 0 ? q.bytes : 1;
  }
  ALDIC_CUDA(cudaMemcpy(m.slab.p, host.data(), upload, cudaMemcpyHostToDevice));
  m.nnz = (long long)col.size();
  m.ninc = (long long)inc.size();
  m.nadj = (long long)acol.size();
  m.device = dev;
  (void)st;
  return OK;
}

constexpr double kQtRtol = 1e-11;
constexpr int kQtMaxit = 50000;

int qt_subpb2(aldic_qt_mesh &m, GridWork &w, double beta, double mu, const double *U,
              const double *F, double *Uhat, cudaStream_t st) {
  int rc;
  if ((rc = qt_upload(m, st))) return rc;
  const int n = m.n, ne = m.ne;
  const double *cx = m.d_coords.as<double>(), *cy = cx + n;
  k_qt_elem<<<nblk(8LL * ne), 256, 0, st>>>(ne, m.d_elems.as<int>(), cx, cy, beta, mu, U, F,
                                            m.d_ke.as<double>(), m.d_be.as<double>());
  k_qt_gather<<<nblk(n), 256, 0, st>>>(n, m.d_iptr.as<int>(), m.d_inc.as<int>(), m.d_ipos.as<int>(),
                                       m.d_row.as<int>(), m.d_ke.as<double>(), m.d_be.as<double>(),
                                       m.d_val.as<double>(), w.b);
  k_qt_elim<<<nblk(n), 256, 0, st>>>(n, m.d_row.as<int>(), m.d_col.as<int>(), m.d_val.as<double>(),
                                     m.d_dpos.as<int>(), m.d_kind.as<unsigned char>(), U, w.b, w.x,
                                     w.mask, m.d_diag.as<double>());
  ALDIC_CUDA(cudaGetLastError());
  const CsrOp op{m.d_row.as<int>(), m.d_col.as<int>(), m.d_val.as<double>(), m.d_diag.as<double>()};
  if ((rc = csr_pcg(w, op, n, 2, kQtRtol, kQtMaxit, st))) return rc;
  k_qt_store<<<nblk(n), 256, 0, st>>>(n, w.x, Uhat);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int qt_subpb2_sweep(aldic_qt_mesh &m, GridWork &w, const double beta[3], double mu,
                    const double *U, const double *F, cudaStream_t st) {
  int rc;
  if ((rc = qt_upload(m, st))) return rc;
  const int n = m.n, ne = m.ne;
  const double *cx = m.d_coords.as<double>(), *cy = cx + n;
  // stiffness part (beta 1, mu 0) into d_val and b fields 0-1, mass part
  // (beta 0, mu 1) into d_valM and b fields 2-3
  for (int part = 0; part < 2; ++part) {
    k_qt_elem<<<nblk(8LL * ne), 256, 0, st>>>(ne, m.d_elems.as<int>(), cx, cy, part ? 0.0 : 1.0,
                                              part ? 1.0 : 0.0, U, F, m.d_ke.as<double>(),
                                              m.d_be.as<double>());
    k_qt_gather<<<nblk(n), 256, 0, st>>>(n, m.d_iptr.as<int>(), m.d_inc.as<int>(),
                                         m.d_ipos.as<int>(), m.d_row.as<int>(), m.d_ke.as<double>(),
                                         m.d_be.as<double>(),
                                         (part ? m.d_valM : m.d_val).as<double>(),
                                         w.b + 2LL * part * n);
  }
  QtBetas be;
  for (int q = 0; q < 3; ++q) be.v[q] = beta[q];
  k_qt_elim3<<<nblk(n), 256, 0, st>>>(n, m.d_row.as<int>(), m.d_col.as<int>(), m.d_val.as<double>(),
                                      m.d_valM.as<double>(), m.d_dpos.as<int>(),
                                      m.d_kind.as<unsigned char>(), U, be, mu, w.b, w.x, w.mask,
                                      m.d_diag.as<double>(), m.d_diagM.as<double>());
  ALDIC_CUDA(cudaGetLastError());
  CsrOp op{m.d_row.as<int>(), m.d_col.as<int>(), m.d_val.as<double>(), m.d_diag.as<double>()};
  op.valM = m.d_valM.as<double>();
  op.diagM = m.d_diagM.as<double>();
  const double be6[6] = {beta[0], beta[0], beta[1], beta[1], beta[2], beta[2]};
  return csr_pcg(w, op, n, 6, kQtRtol, kQtMaxit, st, be6, mu);
}

int qt_store_candidate(aldic_qt_mesh &m, const GridWork &w, int q, double *Uhat, cudaStream_t st) {
  ALDIC_CHECK(q >= 0 && q < 3, E_ARG, "qt_store_candidate: candidate 0..2");
  k_qt_store<<<nblk(m.n), 256, 0, st>>>(m.n, w.x + 2LL * q * m.n, Uhat);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int qt_strain(aldic_qt_mesh &m, const double *U, double *F, cudaStream_t st) {
  int rc;
  if ((rc = qt_upload(m, st))) return rc;
  const int n = m.n, ne = m.ne;
  const double *cx = m.d_coords.as<double>(), *cy = cx + n;
  k_qt_strain_elem<<<nblk(ne), 256, 0, st>>>(ne, m.d_elems.as<int>(), cx, cy, U, m.d_es.as<double>());
  k_qt_strain_gather<<<nblk(n), 256, 0, st>>>(n, m.d_iptr.as<int>(), m.d_inc.as<int>(),
                                              m.d_es.as<double>(), F);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int qt_fill(aldic_qt_mesh &m, GridWork &w, int nf, double *vals, const unsigned char *bad,
            cudaStream_t st) {
  return qt_fill2(m, w, nf, vals, 0, nullptr, bad, st);
}

int qt_fill2(aldic_qt_mesh &m, GridWork &w, int nf1, double *vals1, int nf2, double *vals2,
             const unsigned char *bad, cudaStream_t st) {
  ALDIC_CHECK(nf1 >= 1 && nf2 >= 0 && nf1 + nf2 <= 6 && (nf2 == 0 || vals2), E_ARG,
              "qt_fill: 1..6 fields");
  int rc;
  if ((rc = qt_upload(m, st))) return rc;
  const int n = m.n;
  const int *row = m.d_arow.as<int>(), *col = m.d_acol.as<int>();
  k_qt_fill_prep<<<nblk(n), 256, 0, st>>>(n, nf1, 0, vals1, bad, row, col, w.b, w.x, w.mask);
  if (nf2)
    k_qt_fill_prep<<<nblk(n), 256, 0, st>>>(n, nf2, nf1, vals2, bad, row, col, w.b, w.x, w.mask);
  ALDIC_CUDA(cudaGetLastError());
  const CsrOp op{row, col, m.d_aval.as<double>(), m.d_adiag.as<double>()};
  if ((rc = csr_pcg(w, op, n, nf1 + nf2, kQtRtol, kQtMaxit, st))) return rc;
  k_qt_fill_store<<<nblk(n), 256, 0, st>>>(n, nf1, 0, w.x, bad, vals1);
  if (nf2) k_qt_fill_store<<<nblk(n), 256, 0, st>>>(n, nf2, nf1, w.x, bad, vals2);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

}  // namespace aldic
