// solver.cu -- host orchestration of the AIFMM-LS direct solver on one B200 and
// the C ABI declared in include/aifmm_b200.h.
//
// The control flow follows the reference FMM2DTree (FMM2DTree_find_error.hpp):
//   build tree (:127-1070) -> getNodes (ACA skeletons + L2P/P2M, :1137-1336) ->
//   assemble_M2L (:1338-1361) -> initialise (:1703-1741) ->
//   eliminate_phase_efficient (:2407-2451) -> base solve (:2453-2485) ->
//   back_substitution_phase (:2487-2532).
// All matrix data lives on the device.  The host keeps the block shapes (the
// reference's std::map<int, Mat> bookkeeping) and issues batched launches; it
// waits for the device only where a data-dependent value decides what happens
// next: the ACA ranks of a level, the recompression ranks, and the norms that
// decide which fill-ins are queued for recompression.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "../../include/aifmm_b200.h"
#include "kernels.h"

// geometry / rhs kernels live in k_geom.cu
int aifmm_launch_geometry(int n_cheb, int depth, double L, int q_kind, double q_amp, double q_width, double q_radius,
                          const double* cheb, double2* pts, double* q, double2* leafc, int2* leafxy,
                          cudaStream_t s);
int aifmm_launch_rhs_plane_wave(const double2* pts, const double* q, double kappa, int N, int nrhs,
                                const double* theta, double2* b, cudaStream_t s);
int aifmm_launch_incident_field(const double2* pts, double kappa, int N, int nrhs, const double* theta, double2* u,
                                cudaStream_t s);
int aifmm_launch_gather_segments(const int* src, const int4* segs, long nseg, int* dst, cudaStream_t s);
size_t aifmm_error_norms_scratch_bytes();
int aifmm_launch_error_norms(const double2* x, long ldx, const double2* t, long ldt, long n, int nrhs, double* part,
                             double* out2, cudaStream_t s);
int aifmm_launch_coldot(const double2* a, long lda, const double2* b, long ldb, long n, int nrhs, double2* out,
                        cudaStream_t s);
int aifmm_launch_colaxpby(const double2* x, long ldx, double2* y, long ldy, long n, int nrhs, const double2* alpha,
                          const double2* beta, cudaStream_t s);

namespace {

struct Fail : std::runtime_error {
  aifmm_status st;
  Fail(aifmm_status s, const std::string& m) : std::runtime_error(m), st(s) {}
};

#define CK(call)                                                                                       \
  do {                                                                                                 \
    cudaError_t e__ = (call);                                                                          \
    if (e__ != cudaSuccess)                                                                            \
      throw Fail(e__ == cudaErrorMemoryAllocation ? AIFMM_ERR_NOMEM : AIFMM_ERR_CUDA,                  \
                 std::string(#call) + ": " + cudaGetErrorString(e__) + " (" + __FILE__ + ":" +          \
                     std::to_string(__LINE__) + ")");                                                  \
  } while (0)

#define KL(call)                                                                                       \
  do {                                                                                                 \
    int e__ = (call);                                                                                  \
    ++launches_;                                                                                       \
    if (e__ != 0)                                                                                      \
      throw Fail(AIFMM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString((cudaError_t)e__));   \
  } while (0)

constexpr double2 C1 = {1.0, 0.0};
constexpr double2 CM1 = {-1.0, 0.0};
constexpr double2 C0 = {0.0, 0.0};

// ----------------------------------------------------------------------------
// Device memory: power-of-two size classes carved from large slabs.  Blocks
// released during a box step return to the free lists only after the step, so
// a reused address is always written by a later kernel in stream order.
// ----------------------------------------------------------------------------
class Pool {
 public:
  ~Pool() { release_all(); }
  void* alloc(size_t bytes) {
    if (bytes == 0) return nullptr;
    size_t c = cls(bytes);
    auto& fl = free_[c];
    if (!fl.empty()) { void* p = fl.back(); fl.pop_back(); return p; }
    if (c > (size_t(64) << 20)) {
      void* p = nullptr;
      CK(cudaMalloc(&p, c));
      big_.push_back({p, c});
      return p;
    }
    if (left_ < c) {
      const size_t sz = slab_;
      void* p = nullptr;
      CK(cudaMalloc(&p, sz));
      slabs_.push_back(p);
      slab_bytes_ += sz;
      cur_ = static_cast<char*>(p);
      left_ = sz;
    }
    void* p = cur_;
    cur_ += c;
    left_ -= c;
    return p;
  }
  void defer_free(void* p, size_t bytes) { if (p) pending_.push_back({p, cls(bytes)}); }
  void commit_frees() {
    for (auto& pr : pending_) free_[pr.second].push_back(pr.first);
    pending_.clear();
  }
  void release_all() {
    for (void* p : slabs_) cudaFree(p);
    for (auto& kv : big_) cudaFree(kv.first);
    slabs_.clear(); big_.clear(); free_.clear(); pending_.clear();
    cur_ = nullptr; left_ = 0; slab_bytes_ = 0;
  }
  // slab size: a power of two from 64 MB (the largest block a slab serves) to 512 MB,
  // so that a small problem does not hold half a gigabyte it never uses
  void set_slab(size_t bytes) {
    size_t s = size_t(64) << 20;
    while (s < bytes && s < (size_t(512) << 20)) s <<= 1;
    slab_ = s;
  }
  // return the large blocks that sit in the free lists to the device (the
  // caller has synchronised every stream that used them)
  void release_free_big() {
    for (auto& kv : free_) {
      if (kv.first <= (size_t(64) << 20)) continue;
      for (void* p : kv.second) {
        cudaFree(p);
        for (size_t i = 0; i < big_.size(); ++i)
          if (big_[i].first == p) { big_.erase(big_.begin() + (long)i); break; }
      }
      kv.second.clear();
    }
  }
  size_t reserved() const {
    size_t b = slab_bytes_;
    for (auto& kv : big_) b += kv.second;
    return b;
  }

 private:
  // powers of two up to the slab's largest block, multiples of 64 MB above (a
  // large buffer -- a Krylov basis -- would otherwise round up to twice its size)
  static size_t cls(size_t b) {
    const size_t g = size_t(64) << 20;
    if (b > g) return (b + g - 1) / g * g;
    size_t c = 256;
    while (c < b) c <<= 1;
    return c;
  }
  std::vector<void*> slabs_;
  size_t slab_ = size_t(512) << 20, slab_bytes_ = 0;
  std::vector<std::pair<void*, size_t>> big_;
  std::map<size_t, std::vector<void*>> free_;
  std::vector<std::pair<void*, size_t>> pending_;
  char* cur_ = nullptr;
  size_t left_ = 0;
};

// Bump allocator for per-step scratch (reset when a box step ends).  It starts
// with one chunk sized for the problem and chains further chunks when a step
// needs more; chunks are kept and reused after every reset.
class Arena {
 public:
  void init(size_t bytes) { add_chunk(bytes); }
  ~Arena() { for (auto& c : chunks_) cudaFree(c.first); }
  void* get(size_t bytes) {
    size_t b = (bytes + 255) & ~size_t(255);
    while (cur_ < chunks_.size() && off_ + b > chunks_[cur_].second) { ++cur_; off_ = 0; }
    if (cur_ == chunks_.size()) { add_chunk(std::max(b, chunks_.empty() ? b : chunks_.back().second)); off_ = 0; }
    void* p = chunks_[cur_].first + off_;
    off_ += b;
    return p;
  }
  void reset() { cur_ = 0; off_ = 0; }
  size_t capacity() const {
    size_t s = 0;
    for (auto& c : chunks_) s += c.second;
    return s;
  }

 private:
  void add_chunk(size_t bytes) {
    char* p = nullptr;
    CK(cudaMalloc(&p, bytes));
    chunks_.push_back({p, bytes});
  }
  std::vector<std::pair<char*, size_t>> chunks_;
  size_t cur_ = 0, off_ = 0;
};

// Pinned host + device ring for launch descriptors.  When the ring wraps, the
// copies and kernels that read its older slots must have finished: only the
// handle's own streams use the ring, so those two streams are synchronised
// (never the whole device).
class Staging {
 public:
  void init(size_t bytes, cudaStream_t s1, cudaStream_t s2) {
    CK(cudaMallocHost(&h_, bytes));
    CK(cudaMalloc(&d_, bytes));
    cap_ = bytes;
    s1_ = s1;
    s2_ = s2;
  }
  ~Staging() {
    if (h_) cudaFreeHost(h_);
    if (d_) cudaFree(d_);
  }
  template <class T>
  const T* put(const std::vector<T>& v, cudaStream_t s) { return static_cast<const T*>(put_raw(v.data(), v.size() * sizeof(T), s)); }
  // several arrays in one contiguous region and one copy; returns device pointers
  std::vector<const void*> put_many(std::initializer_list<std::pair<const void*, size_t>> parts, cudaStream_t s) {
    size_t tot = 0;
    for (auto& p : parts) tot += (p.second + 255) & ~size_t(255);
    if (tot > cap_) throw Fail(AIFMM_ERR_NOMEM, "descriptor batch larger than the staging ring");
    if (off_ + tot > cap_) wrap();
    std::vector<const void*> out;
    size_t o = off_;
    for (auto& p : parts) {
      memcpy(h_ + o, p.first, p.second);
      out.push_back(d_ + o);
      o += (p.second + 255) & ~size_t(255);
    }
    CK(cudaMemcpyAsync(d_ + off_, h_ + off_, tot, cudaMemcpyHostToDevice, s));
    off_ += tot;
    return out;
  }
  const void* put_raw(const void* src, size_t bytes, cudaStream_t s) {
    size_t b = (bytes + 255) & ~size_t(255);
    if (b > cap_) throw Fail(AIFMM_ERR_NOMEM, "descriptor batch larger than the staging ring");
    if (off_ + b > cap_) wrap();
    memcpy(h_ + off_, src, bytes);
    CK(cudaMemcpyAsync(d_ + off_, h_ + off_, bytes, cudaMemcpyHostToDevice, s));
    const void* r = d_ + off_;
    off_ += b;
    return r;
  }
  void wrap() {
    if (s1_) CK(cudaStreamSynchronize(s1_));
    if (s2_) CK(cudaStreamSynchronize(s2_));
    off_ = 0;
  }
  char* h_ = nullptr;
  char* d_ = nullptr;
  size_t cap_ = 0, off_ = 0;
  cudaStream_t s1_ = nullptr, s2_ = nullptr;
};

// A device buffer that is kept between calls and grows when a larger one is
// needed (the assembly's per-level ACA workspaces, index lists and LU scratch):
// after the first assemble of a problem size, no call allocates.  Growing waits
// for the handle's stream, so that no kernel still reads the old buffer.
class GrowBuf {
 public:
  ~GrowBuf() { if (p_) cudaFree(p_); }
  void* get(size_t bytes, cudaStream_t s) {
    bytes = std::max<size_t>(bytes, 256);
    if (bytes > cap_) {
      if (p_) {
        CK(cudaStreamSynchronize(s));
        CK(cudaFree(p_));
        p_ = nullptr;
        cap_ = 0;
      }
      const size_t want = std::max(bytes, cap_ + cap_ / 4);
      CK(cudaMalloc(&p_, want));
      cap_ = want;
    }
    return p_;
  }
  size_t capacity() const { return cap_; }
  void release() {  // the caller has synchronised every stream that used the buffer
    if (p_) cudaFree(p_);
    p_ = nullptr;
    cap_ = 0;
  }

 private:
  void* p_ = nullptr;
  size_t cap_ = 0;
};

// A device pointer to complex elements of either form: es = 16 bytes
// (complex128, the assembly and the plain factorisation) or 8 (complex64, the
// factorisation of the mixed form).  Offsets count elements.
struct EP {
  char* b = nullptr;
  int es = 16;
  EP() = default;
  EP(std::nullptr_t) {}
  EP(double2* p) : b(reinterpret_cast<char*>(p)), es(16) {}
  EP(const double2* p) : b(reinterpret_cast<char*>(const_cast<double2*>(p))), es(16) {}
  EP(void* p, int es_) : b(static_cast<char*>(p)), es(es_) {}
  EP operator+(size_t n) const { EP r = *this; if (b) r.b = b + n * (size_t)es; return r; }
  explicit operator bool() const { return b != nullptr; }
  void* v() const { return b; }
  // the complex128 view, for the kernels that exist only in that form
  double2* d() const {
    if (b && es != 16) throw Fail(AIFMM_ERR_STATE, "a complex128 block was expected");
    return reinterpret_cast<double2*>(b);
  }
};

struct Blk {
  EP p;
  int r = 0, c = 0, ld = 0;
  size_t cap = 0;  // bytes owned from the pool (0: view or scratch)
  long size() const { return (long)r * c; }
};

struct QRF {
  Blk qr;
  void* tau = nullptr;          // min(m, n) elements of the factor's type
  int* perm = nullptr;
  int* info = nullptr;
  double* norms = nullptr;
  bool valid = false;
  size_t cap[4] = {0, 0, 0, 0};  // bytes of tau, perm, info, norms owned from the pool (0: scratch)
};

struct Box {
  int nb[8], inner[16], outer[24];
  bool elim = false;
  int NumM = 0, NumL = 0;
  std::vector<int> in_check, in_charge, out_check, out_charge;
  int rank_in = 0, rank_out = 0;
  Blk Ac, Ar, L2P, P2M, L2M_f;
  // Lf[n]: the fill-in L2P_f of neighbour nb[n] formed when this box was
  // eliminated (F:1962-1972); the z-phase and every later solve read it
  Blk Lf[8];
  std::map<int, Blk> M2L, P2P, M2P, P2L, P2M_f, M2M_f;
  // per-solve state: sr the box's particle right-hand side once its
  // smaller-index neighbours are eliminated, sxb = QRx^-1 sr, sy = QRz^-1 (-P2M sxb),
  // smr the multipole right-hand side handed to the parent level
  Blk sr, sxb, sy, smr, particles, multipoles, locals;
  QRF qx, qz;
};

const int NB_DX[8] = {-1, 0, 1, 1, 1, 0, -1, -1};
const int NB_DY[8] = {-1, -1, -1, 0, 1, 1, 1, 0};

int ring_slot(int dx, int dy, int d) {  // ccw position on the ring of radius d from (-d,-d)
  if (dy == -d) return dx + d;
  if (dx == d) return 2 * d + (dy + d);
  if (dy == d) return 4 * d + (d - dx);
  return 6 * d + (d - dy);
}

void box_xy(int k, int level, int& ix, int& iy) {
  ix = iy = 0;
  for (int l = 0; l < level; ++l) {
    int c = (k >> (2 * (level - 1 - l))) & 3;
    ix = 2 * ix + ((c == 1 || c == 2) ? 1 : 0);
    iy = 2 * iy + ((c >= 2) ? 1 : 0);
  }
}
int box_index(int ix, int iy, int level) {
  int k = 0;
  for (int l = level - 1; l >= 0; --l) {
    int bx = (ix >> l) & 1, by = (iy >> l) & 1;
    int c = by ? (bx ? 2 : 3) : (bx ? 1 : 0);
    k = 4 * k + c;
  }
  return k;
}

void gauss_legendre10(double* x, double* w) {  // Newton on P_10, reference ordering (-x,+x by |x|)
  const int n = 10;
  std::vector<std::pair<long double, long double>> r;
  for (int i = 0; i < n / 2; ++i) {
    long double z = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L)), pp = 0;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1, p1 = z;
      for (int k = 2; k <= n; ++k) { long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
      pp = n * (z * p1 - p0) / (z * z - 1);
      long double dz = p1 / pp;
      z -= dz;
      if (fabsl(dz) < 1e-21L) break;
    }
    long double p0 = 1, p1 = z;
    for (int k = 2; k <= n; ++k) { long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
    pp = n * (z * p1 - p0) / (z * z - 1);
    r.push_back({fabsl(z), 2 / ((1 - z * z) * pp * pp)});
  }
  std::sort(r.begin(), r.end());
  for (int i = 0; i < n / 2; ++i) {
    x[2 * i] = (double)(-r[i].first); w[2 * i] = (double)r[i].second;
    x[2 * i + 1] = (double)r[i].first; w[2 * i + 1] = (double)r[i].second;
  }
}

double round6(double v) {  // the reference's Eigen text round trip at stream precision 6
  char buf[64];
  snprintf(buf, sizeof buf, "%.6g", v);
  return strtod(buf, nullptr);
}

}  // namespace

// ============================================================================
struct aifmm_problem {
  aifmm_desc d;
  int device = 0;
  cudaStream_t st = nullptr;
  // second stream for the part of a box step that the step's recompressions do
  // not touch; cur is the stream the batched launches go to
  cudaStream_t st2 = nullptr, cur = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  int rank = 0, N = 0, nleaf = 0, depth = 0, nb = 0;
  double tol = 0;         // ACA (assembly) tolerance, 10^-tol_pow
  double tol_factor = 0;  // recompression tolerance of the factorisation (tol unless set)
  // device geometry and tables
  double2 *d_pts = nullptr, *d_leafc = nullptr, *d_M = nullptr, *d_near = nullptr;
  double* d_q = nullptr;
  int2* d_leafxy = nullptr;
  int* d_iota = nullptr;
  bool tables_ready = false, tree_ready = false, assembled = false;
  // tree
  std::vector<std::vector<Box>> T;
  std::vector<int> nBoxes;
  // memory
  Pool pool;
  Arena scratch;
  Staging stage;
  GrowBuf gb_idx, gb_lst, gb_segs, gb_ws, gb_res, gb_lu, gb_acf;
  // the ACA of a level runs in chunks of boxes whose workspace and factors fit this
  static constexpr size_t kAcaChunkBytes = size_t(2) << 30;
  // timings / counters
  double ms[4] = {0, 0, 0, 0};
  long launches_ = 0, launches_fs = 0, launches_asm = 0;
  int nrhs = 1;
  // pending fill-in candidates of the last eliminated box (kind 0 = P2P, 1 = P2L)
  struct Cand { int kind, nn, pp; };
  std::vector<Cand> cands;
  // Fill-in norm slots in mapped pinned host memory: the norm kernels write them
  // and the host reads them once the event of their phase has completed.
  double* d_norms = nullptr;   // device view of h_norms
  double* h_norms = nullptr;
  int norm_cap = 0;
  cudaEvent_t ev_norm[2] = {nullptr, nullptr};  // after the x- and z-phase norm launches
  int ncand[2] = {0, 0};                        // candidates recorded when each event was set
  bool norms_pending = false;

  EntryCtx ctx() const {
    EntryCtx c;
    c.rank = rank; c.depth = depth; c.kappa = d.kappa;
    c.pts = d_pts; c.q = d_q; c.leafc = d_leafc; c.leafxy = d_leafxy; c.M = d_M; c.nearT = d_near;
    return c;
  }

  // ------------------------------------------------------------------ blocks
  // Element size of the blocks that newblk / scr hand out: 16 (complex128)
  // everywhere except while the mixed form factorises and solves (8, complex64).
  int es_ = 16;
  Blk newblk(int r, int c, int es = 0) {
    if (es == 0) es = es_;
    Blk b; b.r = r; b.c = c; b.ld = r > 0 ? r : 1;
    b.p.es = es;
    if ((long)r * c > 0) { b.cap = (size_t)es * r * c; b.p = EP(pool.alloc(b.cap), es); }
    return b;
  }
  Blk scr(int r, int c, int es = 0) {
    if (es == 0) es = es_;
    Blk b; b.r = r; b.c = c; b.ld = r > 0 ? r : 1;
    b.p.es = es;
    if ((long)r * c > 0) b.p = EP(scratch.get((size_t)es * r * c), es);
    return b;
  }
  void drop(Blk& b) {
    if (b.p && b.cap) pool.defer_free(b.p.v(), b.cap);
    b = Blk();
  }
  void assign(Blk& dst, const Blk& src) { drop(dst); dst = src; }
  // A temporary device buffer from the pool, returned to it when the scope ends
  // (also when an exception leaves the scope); reuse is ordered by the stream.
  struct Tmp {
    aifmm_problem* p; void* ptr; size_t bytes;
    Tmp(aifmm_problem* p_, size_t b) : p(p_), ptr(p_->pool.alloc(std::max<size_t>(b, 1))), bytes(std::max<size_t>(b, 1)) {}
    ~Tmp() { p->pool.defer_free(ptr, bytes); }
    Tmp(const Tmp&) = delete;
    Tmp& operator=(const Tmp&) = delete;
    template <class T> T* as() const { return static_cast<T*>(ptr); }
  };
  void drop_qrf(QRF& f) {
    pool.defer_free(f.tau, f.cap[0]);
    pool.defer_free(f.perm, f.cap[1]);
    pool.defer_free(f.info, f.cap[2]);
    pool.defer_free(f.norms, f.cap[3]);
    f = QRF();
  }

  // ------------------------------------------------------------------ recording
  // While a solve plan is recorded, descriptor arrays go to device blocks owned
  // by the plan (not the staging ring, whose slots are reused) and every launch
  // is also kept as a closure, to be captured into a CUDA graph afterwards.
  bool recording = false;
  std::vector<std::function<int(cudaStream_t)>> rec_ops;
  std::vector<std::pair<void*, size_t>> rec_dev;     // descriptor blocks of the plan being recorded
  std::vector<std::vector<char>> rec_host;           // their host sources, kept until the uploads finish
  std::vector<const void*> put_many_(std::initializer_list<std::pair<const void*, size_t>> parts) {
    if (!recording) return stage.put_many(parts, cur);
    size_t tot = 0;
    for (auto& pr : parts) tot += (pr.second + 255) & ~size_t(255);
    const size_t bytes = std::max<size_t>(tot, 256);
    char* d = static_cast<char*>(pool.alloc(bytes));
    rec_dev.push_back({d, bytes});
    rec_host.emplace_back(tot);
    std::vector<char>& h = rec_host.back();
    std::vector<const void*> out;
    size_t o = 0;
    for (auto& pr : parts) {
      memcpy(h.data() + o, pr.first, pr.second);
      out.push_back(d + o);
      o += (pr.second + 255) & ~size_t(255);
    }
    CK(cudaMemcpyAsync(d, h.data(), tot, cudaMemcpyHostToDevice, cur));
    return out;
  }
  int run_op(std::function<int(cudaStream_t)> f) {
    const int e = f(cur);
    if (recording) rec_ops.push_back(std::move(f));
    return e;
  }

  // ------------------------------------------------------------------ batches
  std::vector<GemmDesc> gd; std::vector<GemmTerm> gt;
  std::vector<GeamDesc> ged;
  std::vector<SolveJob> sj;
  std::vector<QRJob> qj;
  std::vector<FormQJob> fq;
  std::vector<NormDesc> ndv;

  void gemm(const Blk& C, const Blk& A, int opA, const Blk& B, int opB, double2 alpha, double2 beta) {
    const int m = opA ? A.c : A.r, k = opA ? A.r : A.c;
    const int kb = opB ? B.c : B.r, n = opB ? B.r : B.c;
    if (k != kb || C.r != m || C.c != n)
      throw Fail(AIFMM_ERR_NUMERIC, "gemm shape mismatch: C " + std::to_string(C.r) + "x" + std::to_string(C.c) +
                                        " A " + std::to_string(A.r) + "x" + std::to_string(A.c) + " B " +
                                        std::to_string(B.r) + "x" + std::to_string(B.c));
    if (m == 0 || n == 0) return;
    if (k > 0 && (A.p.es != C.p.es || B.p.es != C.p.es))
      throw Fail(AIFMM_ERR_STATE, "gemm operands of different element sizes");
    gemm_batch_es(C.p.es);
    GemmDesc g;
    g.C = C.p.v(); g.ldc = C.ld; g.m = m; g.n = n; g.alpha = alpha; g.beta = beta;
    g.term0 = (int)gt.size(); g.nterms = 0;
    if (k > 0) {
      GemmTerm t; t.A = A.p.v(); t.B = B.p.v(); t.lda = A.ld; t.ldb = B.ld; t.opA = opA; t.opB = opB; t.k = k;
      gt.push_back(t);
      g.nterms = 1;
    }
    gd.push_back(g);
  }
  // C = beta C + alpha * sum_t A_t B_t
  void gemm_sum(const Blk& C, const std::vector<std::pair<Blk, Blk>>& terms, double2 alpha, double2 beta) {
    if (C.r == 0 || C.c == 0) return;
    gemm_batch_es(C.p.es);
    GemmDesc g;
    g.C = C.p.v(); g.ldc = C.ld; g.m = C.r; g.n = C.c; g.alpha = alpha; g.beta = beta;
    g.term0 = (int)gt.size(); g.nterms = 0;
    for (auto& pr : terms) {
      const Blk& A = pr.first; const Blk& B = pr.second;
      if (A.r != C.r || B.c != C.c || A.c != B.r) throw Fail(AIFMM_ERR_NUMERIC, "gemm_sum shape mismatch");
      if (A.c == 0) continue;
      if (A.p.es != C.p.es || B.p.es != C.p.es) throw Fail(AIFMM_ERR_STATE, "gemm operands of different element sizes");
      GemmTerm t; t.A = A.p.v(); t.B = B.p.v(); t.lda = A.ld; t.ldb = B.ld; t.opA = 0; t.opB = 0; t.k = A.c;
      gt.push_back(t);
      ++g.nterms;
    }
    gd.push_back(g);
  }
  // GEMM output-tile width per product shape, set by autotune(): [0] for batches
  // whose products are all thin (n <= 16 columns, e.g. a block times the
  // right-hand sides), [1] otherwise
  int gemm_cols[2] = {32, 32};
  // one element size per batch: a product of the other size flushes the batch first
  int gemm_es = 16;
  void gemm_batch_es(int es) {
    if (!gd.empty() && gemm_es != es) flush_gemm();
    gemm_es = es;
  }
  void flush_gemm() {
    if (gd.empty()) { gt.clear(); return; }
    int nmax = 0;
    for (auto& g : gd) nmax = std::max(nmax, g.n);
    const int tc = gemm_cols[nmax <= 16 ? 0 : 1];
    std::vector<int> off(gd.size());
    int tot = 0;
    for (size_t i = 0; i < gd.size(); ++i) { off[i] = tot; tot += ((gd[i].m + 31) / 32) * ((gd[i].n + tc - 1) / tc); }
    double fl = 0;
    for (auto& g : gd)
      for (int t = 0; t < g.nterms; ++t) fl += 8.0 * g.m * g.n * gt[g.term0 + t].k;
    if (gt.empty()) gt.push_back(GemmTerm{});
    auto ptrs = put_many_({{gt.data(), gt.size() * sizeof(GemmTerm)}, {gd.data(), gd.size() * sizeof(GemmDesc)},
                           {off.data(), off.size() * sizeof(int)}});
    cudaEvent_t a;
    const bool pr = prof_begin(2, a);
    {
      const GemmDesc* d1 = static_cast<const GemmDesc*>(ptrs[1]);
      const GemmTerm* d0 = static_cast<const GemmTerm*>(ptrs[0]);
      const int* d2 = static_cast<const int*>(ptrs[2]);
      const int nd = (int)gd.size(), es = gemm_es;
      KL(run_op([=](cudaStream_t s_) { return aifmm_launch_gemm(d1, d0, d2, nd, tot, s_, tc, es); }));
    }
    if (pr) prof_end(2, a, fl);
    gd.clear(); gt.clear();
  }
  void geam(const Blk& C, const Blk& A, int opA, double2 alpha, double2 beta) {
    const int m = opA ? A.c : A.r, n = opA ? A.r : A.c;
    if (C.r != m || C.c != n) throw Fail(AIFMM_ERR_NUMERIC, "geam shape mismatch");
    if (m == 0 || n == 0) return;
    GeamDesc g; g.A = A.p.v(); g.C = C.p.v(); g.lda = A.ld; g.ldc = C.ld; g.opA = opA; g.m = m; g.n = n;
    g.rs = nullptr; g.cs = nullptr;
    g.esA = A.p.es; g.esC = C.p.es;
    g.alpha = alpha; g.beta = beta;
    ged.push_back(g);
  }
  void copy(const Blk& C, const Blk& A) { geam(C, A, 0, C1, C0); }
  void flush_geam() {
    if (ged.empty()) return;
    std::vector<long long> off(ged.size());
    long long tot = 0;
    for (size_t i = 0; i < ged.size(); ++i) { off[i] = tot; tot += (long long)ged[i].m * ged[i].n; }
    auto ptrs = put_many_({{ged.data(), ged.size() * sizeof(GeamDesc)}, {off.data(), off.size() * sizeof(long long)}});
    {
      const GeamDesc* d0 = static_cast<const GeamDesc*>(ptrs[0]);
      const long long* d1 = static_cast<const long long*>(ptrs[1]);
      const int nd = (int)ged.size();
      KL(run_op([=](cudaStream_t s_) { return aifmm_launch_geam(d0, d1, nd, tot, s_); }));
    }
    ged.clear();
  }
  void zero(const Blk& b) {
    if (b.size() == 0) return;
    if (b.ld == b.r) {
      void* p_ = b.p.v();
      const size_t n_ = (size_t)b.p.es * b.r * b.c;
      CK((cudaError_t)run_op([=](cudaStream_t s_) { return (int)cudaMemsetAsync(p_, 0, n_, s_); }));
    } else {
      for (int j = 0; j < b.c; ++j) {
        void* p_ = (b.p + (size_t)j * b.ld).v();
        const size_t n_ = (size_t)b.p.es * b.r;
        CK((cudaError_t)run_op([=](cudaStream_t s_) { return (int)cudaMemsetAsync(p_, 0, n_, s_); }));
      }
    }
  }
  // QR factorisation of A in place (threshold 0 -> Eigen default)
  void qr_prepare(QRF& f, const Blk& A, double thr, bool persistent) {
    f.qr = A;
    const int n = A.c, s = std::min(A.r, A.c);
    if (persistent) {
      drop_qrf(f);
      f.qr = A;
      f.cap[0] = sizeof(double2) * std::max(1, s);
      f.cap[1] = sizeof(int) * std::max(1, n);
      f.cap[2] = sizeof(int) * 4;
      f.cap[3] = sizeof(double) * std::max(1, 2 * n);
      f.tau = pool.alloc(f.cap[0]);
      f.perm = static_cast<int*>(pool.alloc(f.cap[1]));
      f.info = static_cast<int*>(pool.alloc(f.cap[2]));
      f.norms = static_cast<double*>(pool.alloc(f.cap[3]));
    } else {
      f.tau = scratch.get(sizeof(double2) * std::max(1, s));
      f.perm = static_cast<int*>(scratch.get(sizeof(int) * std::max(1, n)));
      f.info = static_cast<int*>(scratch.get(sizeof(int) * 4));
      f.norms = static_cast<double*>(scratch.get(sizeof(double) * std::max(1, 2 * n)));
    }
    f.valid = true;
    if (!qj.empty() && qr_es != A.p.es) flush_qr();
    qr_es = A.p.es;
    QRJob q; q.a = A.p.v(); q.lda = A.ld; q.m = A.r; q.n = A.c; q.tau = f.tau; q.perm = f.perm; q.norms = f.norms;
    q.thr = thr; q.info = f.info; q.maxpiv = nullptr;
    qj.push_back(q);
  }
  int qr_es = 16, solve_es = 16, formq_es = 16;  // element size of each pending batch
  void flush_qr() {
    if (qj.empty()) return;
    std::vector<QRJob> small, large;
    size_t smem = 0;
    double fl_small = 0, fl_large = 0;
    const int es = qr_es;
    for (auto& j : qj) {
      const size_t b = aifmm_qr_smem_bytes(j.m, j.n, es);
      if (b <= size_t(200) << 10) { small.push_back(j); smem = std::max(smem, b); fl_small += qr_flops(j.m, j.n); }
      else { large.push_back(j); fl_large += qr_flops(j.m, j.n); }
    }
    if (!small.empty()) {
      const QRJob* dq = stage.put(small, cur);
      cudaEvent_t a;
      const bool pr = prof_begin(0, a);
      KL(aifmm_launch_qr_factor_smem(dq, (int)small.size(), smem, es, cur));
      if (pr) prof_end(0, a, fl_small);
    }
    if (!large.empty()) {
      const QRJob* dq = stage.put(large, cur);
      cudaEvent_t a;
      const bool pr = prof_begin(0, a);
      KL(aifmm_launch_qr_factor(dq, (int)large.size(), es, cur));
      if (pr) prof_end(0, a, fl_large);
    }
    qj.clear();
  }
  // X = alpha QR^{-1} B  (B.p == nullptr with B.c = r -> identity)
  void solve(const QRF& f, const Blk& B, const Blk& X, double2 alpha, bool identity = false) {
    const int nr = identity ? X.c : B.c;
    if (!identity && B.r != f.qr.r) throw Fail(AIFMM_ERR_NUMERIC, "solve rhs rows mismatch");
    if (X.r != f.qr.c || X.c != nr) throw Fail(AIFMM_ERR_NUMERIC, "solve output shape mismatch");
    if (nr == 0 || X.r == 0) return;
    const int es = f.qr.p.es;
    if (X.p.es != es || (!identity && B.p.es != es)) throw Fail(AIFMM_ERR_STATE, "solve operands of different element sizes");
    if (!sj.empty() && solve_es != es) flush_solve();
    solve_es = es;
    SolveJob s; s.qr = f.qr.p.v(); s.ldq = f.qr.ld; s.m = f.qr.r; s.n = f.qr.c; s.tau = f.tau; s.perm = f.perm;
    s.info = f.info; s.B = identity ? nullptr : B.p.v(); s.ldb = identity ? 1 : B.ld; s.X = X.p.v(); s.ldx = X.ld;
    s.nrhs = nr; s.alpha = alpha;
    s.work = nullptr;
    sj.push_back(s);
  }
  void flush_solve() {
    if (sj.empty()) return;
    // m <= 224 whose factor fits in shared memory: one warp per column with the
    // column in registers; larger systems (the base level): the global-memory kernel
    std::vector<SolveJob> small, large;
    int mmax = 1, nmax = 1;
    const int es = solve_es;
    for (auto& j : sj) {
      const int s_ = std::min(j.m, j.n);
      const size_t need = (size_t)es * ((size_t)(j.m | 1) * s_ + (size_t)s_) + sizeof(double2) * s_;
      if (j.m <= 224 && need <= (size_t(200) << 10)) {
        small.push_back(j);
        mmax = std::max(mmax, j.m);
        nmax = std::max(nmax, s_);
      } else {
        large.push_back(j);
      }
    }
    if ((size_t)es * ((size_t)(mmax | 1) * nmax + (size_t)nmax) + sizeof(double2) * nmax > (size_t(200) << 10)) {
      // the batch's largest m and rank do not fit together: split by size
      for (auto& j : small) large.push_back(j);
      small.clear();
    }
    if (!small.empty()) {
      std::vector<int> off(small.size());
      int tot = 0;
      for (size_t i = 0; i < small.size(); ++i) { off[i] = tot; tot += (small[i].nrhs + 7) / 8; }
      auto ptrs = put_many_({{small.data(), small.size() * sizeof(SolveJob)}, {off.data(), off.size() * sizeof(int)}});
      double fl = 0;
      for (auto& j : small) { const double mz = std::min(j.m, j.n); fl += (16.0 * j.m * mz - 4.0 * mz * mz) * j.nrhs; }
      cudaEvent_t a;
      const bool pr = prof_begin(1, a);
      {
        const SolveJob* d0 = static_cast<const SolveJob*>(ptrs[0]);
        const int* d1 = static_cast<const int*>(ptrs[1]);
        const int nj = (int)small.size();
        KL(run_op([=](cudaStream_t s_) { return aifmm_launch_qr_solve_warp(d0, d1, nj, tot, mmax, nmax, es, s_); }));
      }
      if (pr) prof_end(1, a, fl);
    }
    if (!large.empty()) {
      std::vector<int> off(large.size());
      int tot = 0;
      for (size_t i = 0; i < large.size(); ++i) {
        off[i] = tot;
        tot += large[i].nrhs;
        large[i].work = scratch.get((size_t)es * large[i].m * large[i].nrhs);
      }
      auto ptrs = put_many_({{large.data(), large.size() * sizeof(SolveJob)}, {off.data(), off.size() * sizeof(int)}});
      double fl = 0;
      for (auto& j : large) { const double mz = std::min(j.m, j.n); fl += (16.0 * j.m * mz - 4.0 * mz * mz) * j.nrhs; }
      cudaEvent_t a;
      const bool pr = prof_begin(1, a);
      {
        const SolveJob* d0 = static_cast<const SolveJob*>(ptrs[0]);
        const int* d1 = static_cast<const int*>(ptrs[1]);
        const int nj = (int)large.size();
        KL(run_op([=](cudaStream_t s_) { return aifmm_launch_qr_solve(d0, d1, nj, tot, es, s_); }));
      }
      if (pr) prof_end(1, a, fl);
    }
    sj.clear();
  }
  void formq(const QRF& f, const Blk& Q) {
    if (Q.size() == 0) return;
    if (Q.p.es != f.qr.p.es) throw Fail(AIFMM_ERR_STATE, "formq operands of different element sizes");
    if (!fq.empty() && formq_es != Q.p.es) flush_formq();
    formq_es = Q.p.es;
    FormQJob j; j.qr = f.qr.p.v(); j.ldq = f.qr.ld; j.m = f.qr.r; j.n = f.qr.c; j.tau = f.tau; j.Q = Q.p.v(); j.ldQ = Q.ld;
    j.ncols_dev = nullptr; j.ncols = Q.c;
    fq.push_back(j);
  }
  void flush_formq() {
    if (fq.empty()) return;
    std::vector<int> off(fq.size());
    int tot = 0;
    for (size_t i = 0; i < fq.size(); ++i) { off[i] = tot; tot += fq[i].ncols; }
    auto ptrs = stage.put_many({{fq.data(), fq.size() * sizeof(FormQJob)}, {off.data(), off.size() * sizeof(int)}}, cur);
    KL(aifmm_launch_formq(static_cast<const FormQJob*>(ptrs[0]), static_cast<const int*>(ptrs[1]), (int)fq.size(),
                          tot, formq_es, cur));
    fq.clear();
  }
  void flush_all() { flush_geam(); flush_qr(); flush_solve(); flush_formq(); flush_gemm(); }
  // Optional CUDA-event timing of selected kernel kinds (aifmm_kernel_profile).
  // kinds: 0 QR factorisation, 1 QR solve, 2 GEMM, 3 ACA, 4 entry blocks, 5 GEAM
  static constexpr int kKinds = 6;
  bool prof_on[kKinds] = {false, false, false, false, false, false};
  struct ProfRec { cudaEvent_t a, b; double flops; };
  std::vector<ProfRec> prof_pending[kKinds];
  std::vector<cudaEvent_t> prof_free;
  long prof_launches[kKinds] = {0, 0, 0, 0, 0, 0};
  double prof_ms[kKinds] = {0, 0, 0, 0, 0, 0}, prof_flops[kKinds] = {0, 0, 0, 0, 0, 0};
  cudaEvent_t prof_event() {
    if (!prof_free.empty()) { cudaEvent_t e = prof_free.back(); prof_free.pop_back(); return e; }
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    return e;
  }
  bool prof_begin(int kind, cudaEvent_t& a) {
    if (!prof_on[kind]) return false;
    a = prof_event();
    CK(cudaEventRecord(a, cur));
    return true;
  }
  void prof_end(int kind, cudaEvent_t a, double flops) {
    cudaEvent_t b = prof_event();
    CK(cudaEventRecord(b, cur));
    prof_pending[kind].push_back({a, b, flops});
    if (prof_pending[kind].size() > 4096) prof_collect();
  }
  void prof_collect() {
    for (int k = 0; k < kKinds; ++k) {
      for (auto& r : prof_pending[k]) {
        CK(cudaEventSynchronize(r.b));
        float ms_ = 0.f;
        CK(cudaEventElapsedTime(&ms_, r.a, r.b));
        prof_ms[k] += ms_;
        prof_flops[k] += r.flops;
        ++prof_launches[k];
        prof_free.push_back(r.a);
        prof_free.push_back(r.b);
      }
      prof_pending[k].clear();
    }
  }
  static double qr_flops(int m, int n) {  // complex Householder QR: 8(m n^2 - n^3/3), m >= n
    const double a = std::max(m, n), b = std::min(m, n);
    return 8.0 * (a * b * b - b * b * b / 3.0);
  }

  // host-side statistics of the last factorize_solve (see aifmm_stats)
  double st_sync_ms = 0, st_compress_ms = 0, st_elim_ms = 0, st_back_ms = 0, st_pending_ms = 0;
  // assembly split: host index lists, ACA (launch to ranks on the host),
  // interpolative operators, M2L/P2P block entries (launch to completion)
  double st_asm_lists_ms = 0, st_asm_aca_ms = 0, st_asm_lu_ms = 0, st_asm_blocks_ms = 0, st_asm_aca_gpu_ms = 0;
  long st_syncs = 0, st_compress = 0, st_apicalls = 0;
  // device -> host read on the handle's stream (never the legacy default stream,
  // which would order this handle against other handles' work)
  void d2h(void* dst, const void* src, size_t bytes) {
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  void sync() {
    auto t0 = std::chrono::steady_clock::now();
    CK(cudaStreamSynchronize(st));
    st_sync_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ++st_syncs;
  }

  // ------------------------------------------------------------------ setup
  void create(const aifmm_desc& desc, int dev) {
    d = desc;
    device = dev;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Fail(AIFMM_ERR_NODEVICE, "no CUDA device");
    if (dev < 0 || dev >= ndev) throw Fail(AIFMM_ERR_ARG, "device index out of range");
    if (d.n_cheb < 2 || d.n_cheb > 16 || d.degree < 1 || d.degree * (d.degree + 1) / 2 > 64 ||
        d.depth < 2 || d.depth > 10 || !(d.L > 0) || !(d.kappa > 0) || d.tol_pow < 1 || d.tol_pow > 15)
      throw Fail(AIFMM_ERR_ARG, "invalid problem description");
    if (d.degree * (d.degree + 1) / 2 > d.n_cheb * d.n_cheb)
      throw Fail(AIFMM_ERR_ARG, "more polynomial bases than nodes per leaf");
    CK(cudaSetDevice(dev));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    cur = st;
    rank = d.n_cheb * d.n_cheb;
    depth = d.depth;
    nleaf = 1 << (2 * depth);
    N = nleaf * rank;
    nb = d.degree * (d.degree + 1) / 2;
    tol = std::pow(10, -1.0 * d.tol_pow);
    tol_factor = tol;
    stage.init(size_t(64) << 20, st, st2);
    pool.set_slab((size_t)N * 2048);  // 512 MB slabs from ~260,000 unknowns up
    // per-step scratch: ~3.6 KB per unknown (2 GB at 589,824 unknowns), at least 64 MB
    scratch.init(std::min(size_t(2) << 30, std::max(size_t(64) << 20, (size_t)N * 3600)));
    CK(cudaMalloc(&d_pts, sizeof(double2) * N));
    CK(cudaMalloc(&d_q, sizeof(double) * N));
    CK(cudaMalloc(&d_leafc, sizeof(double2) * nleaf));
    CK(cudaMalloc(&d_leafxy, sizeof(int2) * nleaf));
    CK(cudaMalloc(&d_M, sizeof(double2) * 121 * rank));
    CK(cudaMalloc(&d_near, sizeof(double2) * 9 * rank * rank));
    CK(cudaMalloc(&d_iota, sizeof(int) * N));
    std::vector<int> iota(N);
    for (int i = 0; i < N; ++i) iota[i] = i;
    CK(cudaMemcpyAsync(d_iota, iota.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    std::vector<double> cheb(d.n_cheb);
    const double PI = 3.1415926535897932384;  // LS_Assembly.hpp:30
    for (int k = 0; k < d.n_cheb; ++k) cheb[k] = -std::cos((k + 0.5) / d.n_cheb * PI);
    const double* d_cheb = static_cast<const double*>(stage.put_raw(cheb.data(), sizeof(double) * cheb.size(), st));
    KL(aifmm_launch_geometry(d.n_cheb, depth, d.L, d.q_kind, d.q_amp, d.q_width, d.q_radius, d_cheb, d_pts, d_q,
                             d_leafc, d_leafxy, st));
    norm_cap = 4096;
    CK(cudaHostAlloc(&h_norms, sizeof(double) * norm_cap, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(&d_norms, h_norms, 0));
    for (auto& e : ev_norm) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    sync();
  }
  void destroy() {
    if (st) cudaStreamSynchronize(st);
    if (st2) cudaStreamSynchronize(st2);
    release_plans();
    pool.release_all();
    cudaFree(d_pts); cudaFree(d_q); cudaFree(d_leafc); cudaFree(d_leafxy); cudaFree(d_M); cudaFree(d_near);
    cudaFree(d_iota);
    if (h_norms) cudaFreeHost(h_norms);
    for (auto& e : ev_norm) if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
    if (st2) cudaStreamDestroy(st2);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
  }

  void tables_compute(int do_round) {
    auto t0 = std::chrono::steady_clock::now();
    double glx[10], glw[10];
    gauss_legendre10(glx, glw);
    std::vector<int2> basis;
    for (int dd = 0; dd < d.degree; ++dd)
      for (int a = 0; a < dd + 1; ++a) basis.push_back(make_int2(a, dd - a));  // LS/FarFieldInteraction.hpp:46-54
    std::vector<double> cheb(d.n_cheb);
    const double PI = 3.1415926535897932384;
    for (int k = 0; k < d.n_cheb; ++k) cheb[k] = -std::cos((k + 0.5) / d.n_cheb * PI);
    double r = d.L;
    for (int j = 0; j < depth; ++j) r = r / 2.0;
    const double* dx = static_cast<const double*>(stage.put_raw(glx, sizeof glx, st));
    const double* dw = static_cast<const double*>(stage.put_raw(glw, sizeof glw, st));
    const int2* db = stage.put(basis, st);
    const double* dc = stage.put(cheb, st);
    Tmp Cw(this, sizeof(double2) * 121 * nb), Vw(this, sizeof(double2) * 9 * rank * nb);
    Tmp status(this, sizeof(int)), qp(this, sizeof(double) * nb * rank);
    CK(cudaMemsetAsync(status.ptr, 0, sizeof(int), st));
    KL(aifmm_launch_tables(d.n_cheb, d.degree, d.kappa, r, dx, dw, db, dc, Cw.as<double2>(), Vw.as<double2>(),
                           status.as<int>(), qp.as<double>(), d_M, d_near, st));
    int h_status = 0;
    CK(cudaMemcpyAsync(&h_status, status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    sync();
    if (h_status) throw Fail(AIFMM_ERR_NUMERIC, "adaptive quadrature exhausted its panel budget");
    if (do_round) {  // the reference's 6-digit text round trip (LS_Assembly.hpp:1178-1228, 1382-1459)
      std::vector<double> M(2 * 121 * rank), Nt(2 * 9 * rank * rank);
      CK(cudaMemcpyAsync(M.data(), d_M, sizeof(double) * M.size(), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(Nt.data(), d_near, sizeof(double) * Nt.size(), cudaMemcpyDeviceToHost, st));
      sync();
      for (double& v : M) v = round6(v);
      for (double& v : Nt) v = round6(v);
      CK(cudaMemcpyAsync(d_M, M.data(), sizeof(double) * M.size(), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(d_near, Nt.data(), sizeof(double) * Nt.size(), cudaMemcpyHostToDevice, st));
      sync();
    }
    pool.commit_frees();
    tables_ready = true;
    ms[1] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  // ------------------------------------------------------------------ tree
  void build_tree() {
    es_ = 16;
    auto t0 = std::chrono::steady_clock::now();
    release_tree();
    T.assign(depth + 1, {});
    nBoxes.assign(depth + 1, 0);
    for (int j = 0; j <= depth; ++j) {
      nBoxes[j] = 1 << (2 * j);
      T[j].assign(nBoxes[j], Box());
      const int n1 = 1 << j;
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& b = T[j][k];
        for (int& v : b.nb) v = -1;
        for (int& v : b.inner) v = -1;
        for (int& v : b.outer) v = -1;
        if (j == 0) continue;
        int x, y;
        box_xy(k, j, x, y);
        for (int dd = 0; dd < 8; ++dd) {
          int nx = x + NB_DX[dd], ny = y + NB_DY[dd];
          if (nx >= 0 && ny >= 0 && nx < n1 && ny < n1) b.nb[dd] = box_index(nx, ny, j);
        }
        if (j < 2) continue;
        const int px = x / 2, py = y / 2;
        for (int ddy = -1; ddy <= 1; ++ddy)
          for (int ddx = -1; ddx <= 1; ++ddx) {
            if (ddx == 0 && ddy == 0) continue;
            const int qx = px + ddx, qy = py + ddy;
            if (qx < 0 || qy < 0 || qx >= n1 / 2 || qy >= n1 / 2) continue;
            for (int cy = 0; cy < 2; ++cy)
              for (int cx = 0; cx < 2; ++cx) {
                const int ox = 2 * qx + cx - x, oy = 2 * qy + cy - y;
                const int dist = std::max(std::abs(ox), std::abs(oy));
                const int id = box_index(2 * qx + cx, 2 * qy + cy, j);
                if (dist == 2) b.inner[ring_slot(ox, oy, 2)] = id;
                else if (dist == 3) b.outer[ring_slot(ox, oy, 3)] = id;
              }
          }
      }
    }
    tree_ready = true;
    assembled = false;
    ms[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  bool well_sep(int j, int k, int l) const {  // F:2077-2088
    if (k == l) return false;
    for (int i = 0; i < 8; ++i) if (T[j][k].nb[i] == l) return false;
    return true;
  }

  // ------------------------------------------------------------------ assembly
  void rows_for(int j, int k, bool in_check, std::vector<int>& out) const {  // F:1182-1228
    if (j == depth) { for (int i = 0; i < rank; ++i) out.push_back(k * rank + i); return; }
    for (int c = 0; c < 4; ++c) {
      const Box& ch = T[j + 1][4 * k + c];
      const auto& v = in_check ? ch.in_check : ch.out_charge;
      out.insert(out.end(), v.begin(), v.end());
    }
  }
  void il_nodes(int j, int k, bool in_check, std::vector<int>& out) const {
    const Box& b = T[j][k];
    for (int i = 0; i < 16; ++i) if (b.inner[i] != -1) rows_for(j, b.inner[i], in_check, out);
    for (int i = 0; i < 24; ++i) if (b.outer[i] != -1) rows_for(j, b.outer[i], in_check, out);
  }

  void assemble() {
    es_ = 16;
    if (!tables_ready) throw Fail(AIFMM_ERR_STATE, "tables not computed or set");
    if (!tree_ready) throw Fail(AIFMM_ERR_STATE, "tree not built");
    auto t0 = std::chrono::steady_clock::now();
    const long l0 = launches_;
    const EntryCtx cx = ctx();
    using clk = std::chrono::steady_clock;
    auto since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
    st_asm_lists_ms = st_asm_aca_ms = st_asm_lu_ms = st_asm_blocks_ms = st_asm_aca_gpu_ms = 0;
    cudaEvent_t ea = nullptr, eb = nullptr;
    CK(cudaEventCreate(&ea));
    CK(cudaEventCreate(&eb));
    for (int j = depth; j >= 2; --j) {
      const int nbx = nBoxes[j];
      auto ta = clk::now();
      // ---- index lists for the outgoing and incoming ACA of every box (F:1230-1336).
      // The point lists of this level's boxes (rows_for) go to the device once; a
      // job's row and column lists are concatenations of them, expanded on the
      // device from a table of (destination, source, length) segments.
      std::vector<int> lst;  // in-lists of all boxes, then out-lists
      std::vector<long> lin_off(nbx + 1), lout_off(nbx + 1);
      for (int k = 0; k < nbx; ++k) { lin_off[k] = (long)lst.size(); rows_for(j, k, true, lst); }
      lin_off[nbx] = (long)lst.size();
      for (int k = 0; k < nbx; ++k) { lout_off[k] = (long)lst.size(); rows_for(j, k, false, lst); }
      lout_off[nbx] = (long)lst.size();
      auto lin_len = [&](int b) { return (int)(lin_off[b + 1] - lin_off[b]); };
      auto lout_len = [&](int b) { return (int)(lout_off[b + 1] - lout_off[b]); };
      std::vector<int> ilb;  // interaction-list boxes of every box: inner, then outer (il_nodes order)
      std::vector<int> ilb_off(nbx + 1);
      for (int k = 0; k < nbx; ++k) {
        ilb_off[k] = (int)ilb.size();
        const Box& B = T[j][k];
        for (int i = 0; i < 16; ++i) if (B.inner[i] != -1) ilb.push_back(B.inner[i]);
        for (int i = 0; i < 24; ++i) if (B.outer[i] != -1) ilb.push_back(B.outer[i]);
      }
      ilb_off[nbx] = (int)ilb.size();
      // point of position rel in the concatenated in-lists (or out-lists) of k's interaction list
      auto il_point = [&](int k, bool in_lists, int rel) {
        for (int q = ilb_off[k]; q < ilb_off[k + 1]; ++q) {
          const int b = ilb[q], len = in_lists ? lin_len(b) : lout_len(b);
          if (rel < len) return lst[(in_lists ? lin_off[b] : lout_off[b]) + rel];
          rel -= len;
        }
        throw Fail(AIFMM_ERR_NUMERIC, "skeleton index outside the interaction list");
      };
      struct JobIdx { long r0, c0; int n1, n2; };
      std::vector<JobIdx> ji(2 * nbx);
      std::vector<int4> segs;
      long cur_i = 0;
      auto seg = [&](long src, int len) {
        if (len > 0) segs.push_back(make_int4((int)cur_i, (int)src, len, 0));
        cur_i += len;
      };
      for (int k = 0; k < nbx; ++k) {
        // outgoing: rows = IL targets (their in-lists), cols = box sources (k's out-list)
        JobIdx& o = ji[2 * k];
        o.r0 = cur_i; o.n1 = 0;
        for (int q = ilb_off[k]; q < ilb_off[k + 1]; ++q) { const int b = ilb[q]; o.n1 += lin_len(b); seg(lin_off[b], lin_len(b)); }
        o.c0 = cur_i; o.n2 = lout_len(k); seg(lout_off[k], o.n2);
        // incoming: rows = box targets (k's in-list), cols = IL sources (their out-lists)
        JobIdx& in = ji[2 * k + 1];
        in.r0 = cur_i; in.n1 = lin_len(k); seg(lin_off[k], in.n1);
        in.c0 = cur_i; in.n2 = 0;
        for (int q = ilb_off[k]; q < ilb_off[k + 1]; ++q) { const int b = ilb[q]; in.n2 += lout_len(b); seg(lout_off[b], lout_len(b)); }
      }
      if (cur_i > INT_MAX || (long)lst.size() > INT_MAX) throw Fail(AIFMM_ERR_NOMEM, "ACA index lists too long");
      int* d_idx = static_cast<int*>(gb_idx.get(sizeof(int) * std::max<long>(1, cur_i), st));
      int* d_lst = static_cast<int*>(gb_lst.get(sizeof(int) * std::max<size_t>(1, lst.size()), st));
      int4* d_segs = static_cast<int4*>(gb_segs.get(sizeof(int4) * std::max<size_t>(1, segs.size()), st));
      if (!lst.empty()) CK(cudaMemcpyAsync(d_lst, lst.data(), sizeof(int) * lst.size(), cudaMemcpyHostToDevice, st));
      if (!segs.empty()) {
        CK(cudaMemcpyAsync(d_segs, segs.data(), sizeof(int4) * segs.size(), cudaMemcpyHostToDevice, st));
        KL(aifmm_launch_gather_segments(d_lst, d_segs, (long)segs.size(), d_idx, st));
      }
      // ---- the level's boxes in chunks: a chunk's ACA workspace and unmodified
      // rows / columns (Ac, Ar: read only by the chunk's interpolative operators)
      // live in reusable buffers of at most kAcaChunkBytes, so the assembly's peak
      // does not grow with the number of boxes of a level.  Every job is computed
      // as in one launch per level.
      auto job_bytes = [&](int t, size_t& wsb, size_t& acb) {
        const int n1 = ji[t].n1, n2 = ji[t].n2, rmax = std::min(n1, n2);
        const int np = n1 < n2 ? n1 : n2, ns = n1 < n2 ? n2 : n1;
        const size_t b = sizeof(double2) * ((size_t)rmax * np + (size_t)rmax * ns + ns + np + 3 * (size_t)rmax + 3) + np + ns + 16;
        wsb = (b + 255) & ~size_t(255);
        acb = (sizeof(double2) * (size_t)rmax * ((t % 2) == 0 ? n2 : n1) + 255) & ~size_t(255);
      };
      st_asm_lists_ms += since(ta);
      for (int k0 = 0; k0 < nbx;) {
        ta = clk::now();
        int k1 = k0;
        size_t ws = 0, acs = 0;
        for (; k1 < nbx; ++k1) {
          size_t w0, a0, w1, a1;
          job_bytes(2 * k1, w0, a0);
          job_bytes(2 * k1 + 1, w1, a1);
          if (k1 > k0 && ws + w0 + w1 + acs + a0 + a1 > kAcaChunkBytes) break;
          ws += w0 + w1;
          acs += a0 + a1;
        }
        const int nch = k1 - k0, nj = 2 * nch, t0 = 2 * k0;
        size_t nres = 0;
        std::vector<size_t> wo(nj), ao(nj), ro(nj);
        {
          size_t w = 0, ac = 0;
          for (int q = 0; q < nj; ++q) {
            size_t wb, ab;
            job_bytes(t0 + q, wb, ab);
            wo[q] = w; w += wb;
            ao[q] = ac; ac += ab;
            ro[q] = nres;
            nres += 2 * (size_t)std::min(ji[t0 + q].n1, ji[t0 + q].n2);
          }
        }
        char* d_ws = static_cast<char*>(gb_ws.get(ws, st));
        char* d_ac = static_cast<char*>(gb_acf.get(acs, st));
        // [2 per job: rank, branch] then the bases
        int* d_res = static_cast<int*>(gb_res.get(sizeof(int) * (2 * (size_t)nj + nres + 1), st));
        int* d_bases = d_res + 2 * nj;
        std::vector<AcaJob> jobs(nj);
        for (int q = 0; q < nj; ++q) {
          const int t = t0 + q, k = t / 2;
          const bool outgoing = (t % 2) == 0;
          const int n1 = ji[t].n1, n2 = ji[t].n2, rmax = std::min(n1, n2);
          const int np = n1 < n2 ? n1 : n2, ns = n1 < n2 ? n2 : n1;
          char* base = d_ws + wo[q];
          AcaJob& J = jobs[q];
          J.rows = d_idx + ji[t].r0; J.cols = d_idx + ji[t].c0; J.n1 = n1; J.n2 = n2;
          J.want_rows = outgoing ? 1 : 0;
          J.U = reinterpret_cast<double2*>(base); base += sizeof(double2) * (size_t)rmax * np;
          J.V = reinterpret_cast<double2*>(base); base += sizeof(double2) * (size_t)rmax * ns;
          J.P = reinterpret_cast<double2*>(base); base += sizeof(double2) * ns;
          J.S = reinterpret_cast<double2*>(base); base += sizeof(double2) * np;
          J.coef = reinterpret_cast<double2*>(base); base += sizeof(double2) * (rmax + 1);
          J.dots_u = reinterpret_cast<double2*>(base); base += sizeof(double2) * (rmax + 1);
          J.dots_v = reinterpret_cast<double2*>(base); base += sizeof(double2) * (rmax + 1);
          J.remP = reinterpret_cast<unsigned char*>(base); base += np;
          J.remS = reinterpret_cast<unsigned char*>(base);
          J.rank = d_res + 2 * q;
          J.prim_bases = d_bases + ro[q];
          J.sec_bases = d_bases + ro[q] + rmax;
          Box& B = T[j][k];
          double2* acp = reinterpret_cast<double2*>(d_ac + ao[q]);
          // views into the chunk buffer (not owned: the next chunk reuses it)
          if (outgoing) { drop(B.Ar); B.Ar = Blk{acp, rmax, n2, std::max(rmax, 1)}; J.out = acp; }
          else { drop(B.Ac); B.Ac = Blk{acp, n1, rmax, std::max(n1, 1)}; J.out = acp; }
        }
        st_asm_lists_ms += since(ta);
        ta = clk::now();
        const AcaJob* dj = stage.put(jobs, st);
        CK(cudaEventRecord(ea, st));
        KL(aifmm_launch_aca(dj, nj, tol, cx, st));
        CK(cudaEventRecord(eb, st));
        // ---- ranks and skeletons back to the host
        std::vector<int> hres(2 * (size_t)nj + nres + 1);
        CK(cudaMemcpyAsync(hres.data(), d_res, sizeof(int) * hres.size(), cudaMemcpyDeviceToHost, st));
        sync();
        std::vector<std::vector<int>> pb(nj), sb(nj);
        std::vector<int> rk(nj), br(nj);
        const int* hb = hres.data() + 2 * nj;
        for (int q = 0; q < nj; ++q) {
          const int rmax = std::min(ji[t0 + q].n1, ji[t0 + q].n2);
          rk[q] = hres[2 * q]; br[q] = hres[2 * q + 1];
          if (rk[q] < 0) throw Fail(AIFMM_ERR_NUMERIC, "ACA block too large");
          pb[q].assign(hb + ro[q], hb + ro[q] + rk[q]);
          sb[q].assign(hb + ro[q] + rmax, hb + ro[q] + rmax + rk[q]);
        }
        {
          float ms_ = 0;
          CK(cudaEventElapsedTime(&ms_, ea, eb));
          st_asm_aca_gpu_ms += ms_;
        }
        st_asm_aca_ms += since(ta);
        ta = clk::now();
        // ---- skeletons, rank equalisation (F:1105-1113) and L2P / P2M jobs
        std::vector<int> sk;  // skeleton index lists for the LU jobs
        struct LUI { long rows, cols; };
        std::vector<LUI> lui(nj);
        for (int k = k0; k < k1; ++k) {
          Box& B = T[j][k];
          const int q0 = 2 * (k - k0);
          B.in_check.clear(); B.in_charge.clear(); B.out_check.clear(); B.out_charge.clear();
          // outgoing (job 2k): rows = the IL boxes' in-lists, cols = k's out-list
          {
            const int q = q0;
            const auto& rb = br[q] == 1 ? pb[q] : sb[q];
            const auto& cb = br[q] == 1 ? sb[q] : pb[q];
            B.rank_out = rk[q];
            for (int r : rb) B.out_check.push_back(il_point(k, true, r));
            for (int c : cb) B.out_charge.push_back(lst[lout_off[k] + c]);
            B.Ar.r = rk[q];
          }
          {
            const int q = q0 + 1;
            const auto& rb = br[q] == 1 ? pb[q] : sb[q];
            const auto& cb = br[q] == 1 ? sb[q] : pb[q];
            B.rank_in = rk[q];
            for (int r : rb) B.in_check.push_back(lst[lin_off[k] + r]);
            for (int c : cb) B.in_charge.push_back(il_point(k, false, c));
            B.Ac.c = rk[q];
          }
          const size_t r = std::min(B.in_check.size(), B.out_check.size());
          B.in_check.resize(r); B.in_charge.resize(r); B.out_check.resize(r); B.out_charge.resize(r);
          lui[q0] = {(long)sk.size(), 0};
          sk.insert(sk.end(), B.in_check.begin(), B.in_check.end());
          lui[q0].cols = (long)sk.size();
          sk.insert(sk.end(), B.in_charge.begin(), B.in_charge.end());
          lui[q0 + 1] = {(long)sk.size(), 0};
          sk.insert(sk.end(), B.out_check.begin(), B.out_check.end());
          lui[q0 + 1].cols = (long)sk.size();
          sk.insert(sk.end(), B.out_charge.begin(), B.out_charge.end());
        }
        const int* d_sk = stage.put(sk.empty() ? std::vector<int>{0} : sk, st);
        std::vector<SkelLUJob> lj;
        size_t lws = 0;
        std::vector<size_t> lwo;
        for (int k = k0; k < k1; ++k) {
          Box& B = T[j][k];
          const int q0 = 2 * (k - k0);
          const int r = (int)B.in_check.size();
          const int m_in = lin_len(k), m_out = lout_len(k);
          drop(B.L2P); drop(B.P2M);
          B.L2P = newblk(m_in, r);
          B.P2M = newblk(r, m_out);
          if (r == 0) continue;
          SkelLUJob a;  // L2P = Ac(:, :r) D1^{-1}, via LU of D1^H (F:1117-1119)
          a.rows = d_sk + lui[q0].rows; a.cols = d_sk + lui[q0].cols; a.r = r; a.adjD = 1;
          a.B = B.Ac.p.d(); a.ldb = B.Ac.ld; a.adjB = 1; a.m = m_in; a.X = B.L2P.p.d(); a.ldx = B.L2P.ld; a.adjX = 1;
          lwo.push_back(lws);
          lws += (sizeof(double2) * ((size_t)r * r + (size_t)r * m_in) + sizeof(int) * r + 511) & ~size_t(255);
          lj.push_back(a);
          SkelLUJob b;  // P2M = D2^{-1} Ar(:r, :) (F:1124-1126)
          b.rows = d_sk + lui[q0 + 1].rows; b.cols = d_sk + lui[q0 + 1].cols; b.r = r; b.adjD = 0;
          b.B = B.Ar.p.d(); b.ldb = B.Ar.ld; b.adjB = 0; b.m = m_out; b.X = B.P2M.p.d(); b.ldx = B.P2M.ld; b.adjX = 0;
          lwo.push_back(lws);
          lws += (sizeof(double2) * ((size_t)r * r + (size_t)r * m_out) + sizeof(int) * r + 511) & ~size_t(255);
          lj.push_back(b);
        }
        if (!lj.empty()) {
          char* d_lw = static_cast<char*>(gb_lu.get(lws, st));
          for (size_t t = 0; t < lj.size(); ++t) {
            char* base = d_lw + lwo[t];
            const int r = lj[t].r, m = lj[t].m;
            lj[t].work = reinterpret_cast<double2*>(base);
            lj[t].piv = reinterpret_cast<int*>(base + sizeof(double2) * ((size_t)r * r + (size_t)r * m));
          }
          const SkelLUJob* dl = stage.put(lj, st);
          KL(aifmm_launch_skel_lu(dl, (int)lj.size(), cx, st));
        }
        sync();  // the chunk buffers are reused by the next chunk
        for (int k = k0; k < k1; ++k) { Box& B = T[j][k]; B.Ac = Blk(); B.Ar = Blk(); }
        pool.commit_frees();
        st_asm_lu_ms += since(ta);
        k0 = k1;
      }
    }
    auto tb = clk::now();
    // ---- M2L blocks (F:1338-1361) and leaf P2P blocks (F:1729-1741)
    {
      std::vector<int> sk;
      std::vector<BlockDesc> bd;
      std::vector<long> rof, cof;  // offsets into sk
      std::vector<std::pair<int, int>> who;  // (level*2^20 + k, kIL)
      std::vector<int> lvl;
      for (int j = 2; j <= depth; ++j) {
        std::vector<long> ic(nBoxes[j]), oc(nBoxes[j]);
        for (int k = 0; k < nBoxes[j]; ++k) {
          ic[k] = (long)sk.size(); sk.insert(sk.end(), T[j][k].in_check.begin(), T[j][k].in_check.end());
          oc[k] = (long)sk.size(); sk.insert(sk.end(), T[j][k].out_charge.begin(), T[j][k].out_charge.end());
        }
        for (int k = 0; k < nBoxes[j]; ++k) {
          Box& B = T[j][k];
          auto add = [&](int kIL) {
            Box& O = T[j][kIL];
            Blk m2l = newblk((int)B.in_check.size(), (int)O.out_charge.size());
            assign(B.M2L[kIL], m2l);
            if (m2l.size() == 0) return;
            BlockDesc x; x.rows = nullptr; x.cols = nullptr; x.nr = m2l.r; x.nc = m2l.c; x.out = m2l.p.d();
            x.ldo = m2l.ld; x.adjoint = 0;
            bd.push_back(x); rof.push_back(ic[k]); cof.push_back(oc[kIL]);
          };
          for (int i = 0; i < 16; ++i) if (B.inner[i] != -1) add(B.inner[i]);
          for (int i = 0; i < 24; ++i) if (B.outer[i] != -1) add(B.outer[i]);
        }
      }
      const int* d_sk = stage.put(sk.empty() ? std::vector<int>{0} : sk, st);
      for (size_t i = 0; i < bd.size(); ++i) { bd[i].rows = d_sk + rof[i]; bd[i].cols = d_sk + cof[i]; }
      for (int k = 0; k < nBoxes[depth]; ++k) {
        Box& B = T[depth][k];
        auto add = [&](int nn) {
          Blk p = newblk(rank, rank);
          assign(B.P2P[nn], p);
          BlockDesc x; x.rows = d_iota + (size_t)k * rank; x.cols = d_iota + (size_t)nn * rank; x.nr = rank;
          x.nc = rank; x.out = p.p.d(); x.ldo = rank; x.adjoint = 0;
          bd.push_back(x);
        };
        for (int n = 0; n < 8; ++n) if (B.nb[n] != -1) add(B.nb[n]);
        add(k);
      }
      launch_blocks(bd);
    }
    // ---- initialise_phase (F:1714-1727)
    for (int j = 2; j <= depth; ++j)
      for (int k = 0; k < nBoxes[j]; ++k) { Box& B = T[j][k]; B.NumM = B.P2M.r; B.NumL = B.L2P.c; }
    sync();
    st_asm_blocks_ms = since(tb);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    pool.commit_frees();
    assembled = true;
    launches_asm = launches_ - l0;
    ms[2] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  void launch_blocks(const std::vector<BlockDesc>& bd) {
    if (bd.empty()) return;
    std::vector<long long> off(bd.size());
    long long tot = 0;
    for (size_t i = 0; i < bd.size(); ++i) { off[i] = tot; tot += (long long)bd[i].nr * bd[i].nc; }
    auto ptrs = stage.put_many({{bd.data(), bd.size() * sizeof(BlockDesc)}, {off.data(), off.size() * sizeof(long long)}}, st);
    KL(aifmm_launch_block_entries(static_cast<const BlockDesc*>(ptrs[0]), static_cast<const long long*>(ptrs[1]),
                                  (int)bd.size(), tot, ctx(), st));
  }

  // ------------------------------------------------------------------ elimination
  Blk& X_of(Box& Nn, bool nn_elim, int k) { return nn_elim ? Nn.P2L[k] : Nn.P2P[k]; }

  void record_cand(int kind, int nn, int pp, const Blk& b) {
    if ((int)cands.size() >= norm_cap) throw Fail(AIFMM_ERR_NUMERIC, "too many fill-in candidates");
    // every slot is written by a norm kernel (an empty block gives 0), so all
    // writes to the slots are ordered by the stream
    NormDesc n; n.A = b.p.v(); n.es = b.p.es; n.lda = std::max(b.ld, 1); n.m = b.size() ? b.r : 0; n.n = b.size() ? b.c : 0;
    n.out = d_norms + cands.size();
    cands.push_back({kind, nn, pp});
    ndv.push_back(n);
  }
  // phase 0: the norms recorded by eliminate_x; phase 1: by eliminate_z
  void flush_norms(int phase) {
    if (!ndv.empty()) {
      const NormDesc* dn = stage.put(ndv, st);
      KL(aifmm_launch_norms(dn, (int)ndv.size(), st));
      ndv.clear();
    }
    CK(cudaEventRecord(ev_norm[phase], st));
    ncand[phase] = (int)cands.size();
  }
  void wait_norms(int phase) {
    auto t0 = std::chrono::steady_clock::now();
    CK(cudaEventSynchronize(ev_norm[phase]));
    st_sync_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ++st_syncs;
  }
  void clear_cands() { cands.clear(); ncand[0] = ncand[1] = 0; }

  // The part of eliminate_x that the recompressions of the same step cannot
  // change: they touch the bases of k and of boxes well separated from k, the
  // M2L blocks and the level above, never P2P[k][k], k's right-hand side or its
  // blocks towards its neighbours.  So the factorisation of P2P[k][k] and its
  // solves with those blocks run on the second stream, overlapping the
  // recompressions and their synchronisations on the main stream.
  struct SideX { bool on = false; Blk W[8]; };
  SideX sx;
  void eliminate_x_side(int j, int k) {
    sx = SideX();
    Box& B = T[j][k];
    Blk& Pkk = B.P2P[k];
    if (Pkk.size() == 0) return;
    flush_all();
    CK(cudaEventRecord(ev_fork, st));
    CK(cudaStreamWaitEvent(st2, ev_fork, 0));
    cur = st2;
    qr_prepare(B.qx, Pkk, 0.0, true);  // factored in place; P2P[k][k] is not read again
    flush_qr();
    const int m = Pkk.c;
    for (int pI = 0; pI < 8; ++pI) {
      const int pp = B.nb[pI];
      if (pp == -1) continue;
      const Blk& src = T[j][pp].elim ? B.M2P[pp] : B.P2P[pp];
      sx.W[pI] = scr(m, src.c);
      solve(B.qx, src, sx.W[pI], C1);
    }
    flush_solve();
    CK(cudaEventRecord(ev_join, st2));
    cur = st;
    sx.on = true;
  }
  void eliminate_x(int j, int k) {  // F:1814-1840, 1961-2075 (and the no-QR branch :1843-1957)
    Box& B = T[j][k];
    Blk& Pkk = B.P2P[k];
    if (Pkk.size() != 0) {
      const int m = Pkk.c;
      Blk XL = scr(m, B.L2P.c), W[8];
      if (sx.on) {
        CK(cudaStreamWaitEvent(st, ev_join, 0));
        for (int q = 0; q < 8; ++q) W[q] = sx.W[q];
        solve(B.qx, B.L2P, XL, C1);
      } else {
        qr_prepare(B.qx, Pkk, 0.0, true);
        flush_qr();
        solve(B.qx, B.L2P, XL, C1);
        for (int pI = 0; pI < 8; ++pI) {
          const int pp = B.nb[pI];
          if (pp == -1) continue;
          const Blk& src = T[j][pp].elim ? B.M2P[pp] : B.P2P[pp];
          W[pI] = scr(m, src.c);
          solve(B.qx, src, W[pI], C1);
        }
      }
      sx.on = false;
      flush_solve();
      { Blk t = newblk(B.P2M.r, XL.c); gemm(t, B.P2M, 0, XL, 0, CM1, C0); assign(B.L2M_f, t); }
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        Blk t = newblk(B.P2M.r, W[n].c);
        gemm(t, B.P2M, 0, W[n], 0, CM1, C0);
        if (!T[j][nn].elim) assign(B.P2M_f[nn], t); else assign(B.M2M_f[nn], t);
      }
      // box k's own products first: the z-phase factorisation and solves need only
      // them, and run on the second stream while the fill-ins of the neighbours'
      // blocks below are computed
      flush_gemm();
      eliminate_z_side(j, k);
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        Box& Nn = T[j][nn];
        const Blk Xnk = X_of(Nn, Nn.elim, k);
        { Blk t = newblk(Xnk.r, XL.c); gemm(t, Xnk, 0, XL, 0, CM1, C0); assign(B.Lf[n], t); }
        for (int pI = 0; pI < 8; ++pI) {
          const int pp = B.nb[pI];
          if (pp == -1) continue;
          const bool pe = T[j][pp].elim;
          Blk* tgt;
          int kind = -1;
          if (!Nn.elim) { tgt = pe ? &Nn.M2P[pp] : &Nn.P2P[pp]; if (!pe && well_sep(j, nn, pp) && nn < pp) kind = 0; }
          else { tgt = pe ? &Nn.M2L[pp] : &Nn.P2L[pp]; if (!pe && well_sep(j, nn, pp)) kind = 1; }
          const bool must_exist = Nn.elim && pe;  // M2L: the reference subtracts without a size check
          if (tgt->size() == 0 && !must_exist) {
            Blk t = newblk(Xnk.r, W[pI].c);
            gemm(t, Xnk, 0, W[pI], 0, CM1, C0);
            assign(*tgt, t);
          } else {
            gemm(*tgt, Xnk, 0, W[pI], 0, CM1, C1);
          }
          if (kind >= 0) record_cand(kind, nn, pp, *tgt);
        }
      }
      flush_gemm();
      flush_norms(0);
    } else {
      // box k carries no unknowns: the reference stores uninitialised blocks whose
      // intended value (a product with an empty inner dimension) is zero
      { Blk t = newblk(B.P2M.r, B.L2P.c); zero(t); assign(B.L2M_f, t); }
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        if (!T[j][nn].elim) { Blk t = newblk(B.P2M.r, B.P2P[nn].c); zero(t); assign(B.P2M_f[nn], t); }
        else { Blk t = newblk(B.P2M.r, B.M2P[nn].c); zero(t); assign(B.M2M_f[nn], t); }
      }
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        Box& Nn = T[j][nn];
        { Blk t = newblk(X_of(Nn, Nn.elim, k).r, B.L2P.c); zero(t); assign(B.Lf[n], t); }
        for (int pI = 0; pI < 8; ++pI) {
          const int pp = B.nb[pI];
          if (pp == -1) continue;
          const bool pe = T[j][pp].elim;
          if (!Nn.elim) {
            if (!pe) {
              Blk& t = Nn.P2P[pp];
              if (t.size() == 0) { Blk z = newblk(Nn.P2P[k].r, B.P2P[pp].c); zero(z); assign(t, z); }
              if (well_sep(j, nn, pp) && nn < pp) record_cand(0, nn, pp, t);
            } else {
              Blk& t = Nn.M2P[pp];
              if (t.size() == 0) { Blk z = newblk(Nn.P2P[k].r, B.M2P[pp].c); zero(z); assign(t, z); }
            }
          } else if (!pe) {
            Blk& t = Nn.P2L[pp];
            if (t.size() == 0) { Blk z = newblk(Nn.P2L[k].r, B.P2P[pp].c); zero(z); assign(t, z); }
            if (well_sep(j, nn, pp)) record_cand(1, nn, pp, t);
          }
        }
      }
      flush_norms(0);
    }
  }

  // The factorisation of L2M_f and its solves (F:2090-2113, 2245-2279): they read
  // L2M_f, P2M_f / M2M_f and the local right-hand side of box k and write only k's
  // own blocks, while the x-phase fill-ins write only the neighbours' blocks.
  bool sz_on = false;
  void eliminate_z_qr_solves(int j, int k) {
    Box& B = T[j][k];
    qr_prepare(B.qz, B.L2M_f, 0.0, true);
    flush_qr();
    const int nl = B.L2M_f.c;
    { Blk t = newblk(nl, B.NumM); solve(B.qz, Blk(), t, CM1, true); assign(B.M2L[k], t); }  // QR2^{-1}(-I)
    for (int n = 0; n < 8; ++n) {
      const int nn = B.nb[n];
      if (nn == -1) continue;
      if (!T[j][nn].elim) { Blk t = newblk(nl, B.P2M_f[nn].c); solve(B.qz, B.P2M_f[nn], t, C1); assign(B.P2L[nn], t); }
      else { Blk t = newblk(nl, B.M2M_f[nn].c); solve(B.qz, B.M2M_f[nn], t, C1); assign(B.M2L[nn], t); }
      // well-separated test of (k, nn) is false for a neighbour: nothing is queued here
    }
    flush_solve();
  }
  void eliminate_z_side(int j, int k) {
    sz_on = false;
    if (T[j][k].L2M_f.size() == 0) return;
    flush_all();
    CK(cudaEventRecord(ev_fork, st));
    CK(cudaStreamWaitEvent(st2, ev_fork, 0));
    cur = st2;
    eliminate_z_qr_solves(j, k);
    CK(cudaEventRecord(ev_join, st2));
    cur = st;
    sz_on = true;
  }
  void eliminate_z(int j, int k) {  // F:2090-2113, 2245-2372 (and the no-QR branch :2116-2242)
    Box& B = T[j][k];
    if (B.L2M_f.size() > 0) {
      if (sz_on) CK(cudaStreamWaitEvent(st, ev_join, 0));
      else eliminate_z_qr_solves(j, k);
      sz_on = false;
      const Blk Yneg = B.M2L[k];
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        Box& Nn = T[j][nn];
        const Blk Lf = B.Lf[n];
        {  // F:2348-2372
          Blk& tgt = Nn.elim ? Nn.M2L[k] : Nn.M2P[k];
          if (tgt.size() == 0) { Blk t = newblk(Lf.r, Yneg.c); gemm(t, Lf, 0, Yneg, 0, CM1, C0); assign(tgt, t); }
          else gemm(tgt, Lf, 0, Yneg, 0, CM1, C1);
        }
        for (int pI = 0; pI < 8; ++pI) {  // F:2296-2346
          const int pp = B.nb[pI];
          if (pp == -1) continue;
          const bool pe = T[j][pp].elim;
          const Blk Z = pe ? B.M2L[pp] : B.P2L[pp];
          Blk* tgt;
          int kind = -1;
          if (!Nn.elim) { tgt = pe ? &Nn.M2P[pp] : &Nn.P2P[pp]; if (!pe && well_sep(j, nn, pp) && nn < pp) kind = 0; }
          else { tgt = pe ? &Nn.M2L[pp] : &Nn.P2L[pp]; if (!pe && well_sep(j, nn, pp)) kind = 1; }
          gemm(*tgt, Lf, 0, Z, 0, CM1, C1);
          if (kind >= 0) record_cand(kind, nn, pp, *tgt);
        }
      }
      flush_gemm();
      flush_norms(1);
    } else {
      { Blk t = newblk(0, B.NumM); assign(B.M2L[k], t); }
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        if (!T[j][nn].elim) { Blk t = newblk(0, B.P2M_f[nn].c); assign(B.P2L[nn], t); }
        else { Blk t = newblk(0, B.M2M_f[nn].c); assign(B.M2L[nn], t); }
      }
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        Box& Nn = T[j][nn];
        Blk& tgt = Nn.elim ? Nn.M2L[k] : Nn.M2P[k];
        if (tgt.size() == 0) { Blk t = newblk(B.Lf[n].r, B.NumM); zero(t); assign(tgt, t); }
        for (int pI = 0; pI < 8; ++pI) {
          const int pp = B.nb[pI];
          if (pp == -1) continue;
          const bool pe = T[j][pp].elim;
          if (!Nn.elim && !pe) { if (well_sep(j, nn, pp) && nn < pp) record_cand(0, nn, pp, Nn.P2P[pp]); }
          else if (Nn.elim && !pe) { if (well_sep(j, nn, pp)) record_cand(1, nn, pp, Nn.P2L[pp]); }
        }
      }
      flush_norms(1);
    }
  }

  // ---- recompression (F:1424-1699)
  struct CompressOut { Blk nL, nPt, M2L; };
  // Both directions in one launch of the fused kernel (one CTA each), then one
  // synchronisation to read the four ranks.  Returns false, having enqueued
  // nothing, when a direction's working set does not fit in shared memory.
  bool compress_P2P_pair_fused(int j, int k, int b, CompressOut& kb, CompressOut& bk) {
    const int kk[2] = {k, b}, bb[2] = {b, k};
    CompressOut* out[2] = {&kb, &bk};
    size_t smem = 0;
    for (int s = 0; s < 2; ++s) {
      Box& K = T[j][kk[s]];
      Box& Bb = T[j][bb[s]];
      const Blk& Pkb = K.P2P[bb[s]];
      const Blk& m2l = K.M2L[bb[s]];
      if (Pkb.r != K.L2P.r) throw Fail(AIFMM_ERR_NUMERIC, "compress_P2P: block rows mismatch");
      if (Bb.P2M.c != Pkb.c || m2l.r != K.L2P.c || m2l.c != Bb.P2M.r)
        throw Fail(AIFMM_ERR_NUMERIC, "compress_P2P: block shapes");
      const size_t need = aifmm_compress_smem_bytes(K.L2P.r, K.L2P.c, Pkb.c, Bb.P2M.r, es_);
      if (need == 0) return false;
      smem = std::max(smem, need);
    }
    std::vector<CompressJob> jobs(2);
    int* ranks = static_cast<int*>(scratch.get(sizeof(int) * 4));
    int rcmax[2], rrmax[2];
    for (int s = 0; s < 2; ++s) {
      Box& K = T[j][kk[s]];
      Box& Bb = T[j][bb[s]];
      const Blk& Pkb = K.P2P[bb[s]];
      const Blk& m2l = K.M2L[bb[s]];
      const int m = K.L2P.r, rK = K.L2P.c, c = Pkb.c, rb = Bb.P2M.r, n1 = rK + c;
      rcmax[s] = std::min(m, n1);
      const int n2max = rb + rcmax[s];
      rrmax[s] = std::min(c, n2max);
      out[s]->nL = newblk(m, rcmax[s]);
      out[s]->nPt = newblk(c, rrmax[s]);
      out[s]->M2L = scr(rcmax[s], rrmax[s]);
      CompressJob& J = jobs[s];
      for (const Blk* x : std::initializer_list<const Blk*>{&K.L2P, &Pkb, &Bb.P2M, &m2l})
        if (x->size() && x->p.es != es_) throw Fail(AIFMM_ERR_STATE, "compress_P2P: block of the other form");
      J.L2P = K.L2P.p.v(); J.ldL = K.L2P.ld;
      J.Pkb = Pkb.p.v(); J.ldP = Pkb.ld;
      J.P2M = Bb.P2M.p.v(); J.ldM = Bb.P2M.ld;
      J.M2L = m2l.p.v(); J.ldT = m2l.ld;
      J.m = m; J.rK = rK; J.c = c; J.rb = rb; J.tol = tol_factor;
      J.nL = out[s]->nL.p.v(); J.nPt = out[s]->nPt.p.v();
      J.M2Lo = out[s]->M2L.p.v(); J.ldO = out[s]->M2L.ld;
      J.ranks = ranks + 2 * s;
      auto cg = [&](long elems) { return scratch.get((size_t)es_ * std::max(1L, elems)); };
      J.Acol = cg((long)m * n1);
      J.Arow = cg((long)c * n2max);
      J.tau = cg(std::max(rcmax[s], rrmax[s]));
      J.perm = static_cast<int*>(scratch.get(sizeof(int) * std::max(1, std::max(n1, n2max))));
      J.info = static_cast<int*>(scratch.get(sizeof(int) * 4));
      J.Rkp = cg((long)rcmax[s] * c);
      J.Rk = cg((long)rcmax[s] * rK);
      J.Rn = cg((long)rrmax[s] * rb);
      J.Rnp = cg((long)rrmax[s] * rcmax[s]);
      J.Tm = cg((long)rcmax[s] * rb);
    }
    flush_all();
    const CompressJob* dj = stage.put(jobs, st);
    KL(aifmm_launch_compress_p2p(dj, 2, smem, es_, st));
    sync();
    int rk[4];
    d2h(rk, ranks, sizeof rk);
    for (int s = 0; s < 2; ++s) {
      const int rc = rk[2 * s], rr = rk[2 * s + 1];
      if (rc < 0 || rc > rcmax[s] || rr < 0 || rr > rrmax[s]) throw Fail(AIFMM_ERR_NUMERIC, "compress_P2P: rank out of range");
      out[s]->nL.c = rc;
      out[s]->nPt.c = rr;
      out[s]->M2L.r = rc;
      out[s]->M2L.c = rr;
    }
    return true;
  }
  // Both directions of compress_P2P (F:1532-1559) in lockstep: (k,b) and (b,k)
  void compress_P2P_pair(int j, int k, int b, CompressOut& kb, CompressOut& bk) {
    if (compress_P2P_pair_fused(j, k, b, kb, bk)) return;
    int kk[2] = {k, b}, bb[2] = {b, k};
    Blk Acol[2], Rk_prime[2], Rk[2], Arow[2];
    QRF qc[2], qw[2];
    int rc[2], rr[2];
    CompressOut* out[2] = {&kb, &bk};
    for (int s = 0; s < 2; ++s) {
      Box& K = T[j][kk[s]];
      const Blk& Pkb = K.P2P[bb[s]];
      if (Pkb.r != K.L2P.r) throw Fail(AIFMM_ERR_NUMERIC, "compress_P2P: block rows mismatch");
      Acol[s] = scr(K.L2P.r, K.L2P.c + Pkb.c);
      copy(Blk{Acol[s].p, K.L2P.r, K.L2P.c, Acol[s].ld}, K.L2P);
      copy(Blk{Acol[s].p + (size_t)K.L2P.c * Acol[s].ld, Pkb.r, Pkb.c, Acol[s].ld}, Pkb);
    }
    flush_geam();
    for (int s = 0; s < 2; ++s) qr_prepare(qc[s], Acol[s], tol_factor, false);
    flush_qr();
    sync();
    for (int s = 0; s < 2; ++s) {
      int info[2];
      d2h(info, qc[s].info, sizeof info);
      rc[s] = info[1];
    }
    for (int s = 0; s < 2; ++s) {
      out[s]->nL = newblk(Acol[s].r, rc[s]);
      formq(qc[s], out[s]->nL);
    }
    flush_formq();
    for (int s = 0; s < 2; ++s) {
      Box& K = T[j][kk[s]];
      const Blk& Pkb = K.P2P[bb[s]];
      Rk_prime[s] = scr(rc[s], Pkb.c);
      Rk[s] = scr(rc[s], K.L2P.c);
      gemm(Rk_prime[s], out[s]->nL, 1, Pkb, 0, C1, C0);
      gemm(Rk[s], out[s]->nL, 1, K.L2P, 0, C1, C0);
    }
    flush_gemm();
    for (int s = 0; s < 2; ++s) {
      Box& Bb = T[j][bb[s]];
      const int mb = Bb.P2M.c, rb = Bb.P2M.r;
      Arow[s] = scr(mb, rb + rc[s]);
      geam(Blk{Arow[s].p, mb, rb, Arow[s].ld}, Bb.P2M, 1, C1, C0);
      geam(Blk{Arow[s].p + (size_t)rb * Arow[s].ld, mb, rc[s], Arow[s].ld}, Rk_prime[s], 1, C1, C0);
    }
    flush_geam();
    for (int s = 0; s < 2; ++s) qr_prepare(qw[s], Arow[s], tol_factor, false);
    flush_qr();
    sync();
    for (int s = 0; s < 2; ++s) {
      int info[2];
      d2h(info, qw[s].info, sizeof info);
      rr[s] = info[1];
    }
    for (int s = 0; s < 2; ++s) {
      out[s]->nPt = newblk(Arow[s].r, rr[s]);
      formq(qw[s], out[s]->nPt);
    }
    flush_formq();
    Blk Rn[2], Rnp[2], Tm[2];
    for (int s = 0; s < 2; ++s) {
      Box& K = T[j][kk[s]];
      Box& Bb = T[j][bb[s]];
      Rn[s] = scr(rr[s], Bb.P2M.r);
      Rnp[s] = scr(rr[s], rc[s]);
      gemm(Rn[s], out[s]->nPt, 1, Bb.P2M, 1, C1, C0);
      gemm(Rnp[s], out[s]->nPt, 1, Rk_prime[s], 1, C1, C0);
      const Blk& m2l = K.M2L[bb[s]];
      if (m2l.r != Rk[s].c || m2l.c != Bb.P2M.r) throw Fail(AIFMM_ERR_NUMERIC, "compress_P2P: M2L shape");
      Tm[s] = scr(rc[s], m2l.c);
      gemm(Tm[s], Rk[s], 0, m2l, 0, C1, C0);
    }
    flush_gemm();
    for (int s = 0; s < 2; ++s) {
      out[s]->M2L = scr(rc[s], rr[s]);
      gemm(out[s]->M2L, Tm[s], 0, Rn[s], 1, C1, C0);
    }
    flush_gemm();
    for (int s = 0; s < 2; ++s) geam(out[s]->M2L, Rnp[s], 1, C1, C1);
    flush_geam();
  }

  // Tk = nL^H L2P_k  (new locals from old)
  void update_other_M2Ls_at_k(int j, int k, int b, const Blk& Tk) {  // F:1594-1630
    Box& K = T[j][k];
    auto upd = [&](int x) {
      Blk& m = K.M2L[x];
      Blk t = newblk(Tk.r, m.c);
      gemm(t, Tk, 0, m, 0, C1, C0);
      assign(m, t);
    };
    for (int i = 0; i < 16; ++i) if (K.inner[i] != -1 && K.inner[i] != b) upd(K.inner[i]);
    for (int i = 0; i < 24; ++i) if (K.outer[i] != -1 && K.outer[i] != b) upd(K.outer[i]);
    for (int n = 0; n < 8; ++n) { int kN = K.nb[n]; if (kN != -1 && T[j][kN].elim && K.elim) upd(kN); }
    if (K.elim) upd(k);
  }
  // Tb = P2M_b nPt (old multipoles to new)
  void update_other_M2Ls_at_b(int j, int k, int b, const Blk& Tb) {  // F:1632-1669
    Box& Bb = T[j][b];
    auto upd = [&](int x) {
      Blk& m = T[j][x].M2L[b];
      Blk t = newblk(m.r, Tb.c);
      gemm(t, m, 0, Tb, 0, C1, C0);
      assign(m, t);
    };
    for (int i = 0; i < 16; ++i) if (Bb.inner[i] != -1 && Bb.inner[i] != k) upd(Bb.inner[i]);
    for (int i = 0; i < 24; ++i) if (Bb.outer[i] != -1 && Bb.outer[i] != b) upd(Bb.outer[i]);  // as in the reference
    for (int n = 0; n < 8; ++n) { int kN = Bb.nb[n]; if (kN != -1 && T[j][kN].elim && Bb.elim) upd(kN); }
    if (Bb.elim) upd(b);
  }
  void update_parent_L2P(int j, int k, const Blk& Tk) {  // F:1671-1684
    const int kP = k / 4, ck = k % 4;
    Box& P = T[j - 1][kP];
    int off[5] = {0, 0, 0, 0, 0};
    for (int c = 0; c < 4; ++c) off[c + 1] = off[c] + T[j][kP * 4 + c].NumL;
    const int tot = off[4] - T[j][k].NumL + Tk.r;
    Blk np = newblk(tot, P.L2P.c);
    int o = 0;
    for (int c = 0; c < 4; ++c) {
      const int nl = T[j][kP * 4 + c].NumL;
      Blk src{P.L2P.p + off[c], nl, P.L2P.c, P.L2P.ld};
      if (c == ck) {
        gemm(Blk{np.p + o, Tk.r, np.c, np.ld}, Tk, 0, src, 0, C1, C0);
        o += Tk.r;
      } else {
        copy(Blk{np.p + o, nl, np.c, np.ld}, src);
        o += nl;
      }
    }
    assign(P.L2P, np);
  }
  void update_parent_P2M(int j, int b, const Blk& Tb) {  // F:1686-1699
    const int bP = b / 4, cb = b % 4;
    Box& P = T[j - 1][bP];
    int off[5] = {0, 0, 0, 0, 0};
    for (int c = 0; c < 4; ++c) off[c + 1] = off[c] + T[j][bP * 4 + c].NumM;
    const int tot = off[4] - T[j][b].NumM + Tb.c;
    Blk np = newblk(P.P2M.r, tot);
    int o = 0;
    for (int c = 0; c < 4; ++c) {
      const int nm = T[j][bP * 4 + c].NumM;
      Blk src{P.P2M.p + (size_t)off[c] * P.P2M.ld, P.P2M.r, nm, P.P2M.ld};
      if (c == cb) {
        gemm(Blk{np.p + (size_t)o * np.ld, np.r, Tb.c, np.ld}, src, 0, Tb, 0, C1, C0);
        o += Tb.c;
      } else {
        copy(Blk{np.p + (size_t)o * np.ld, np.r, nm, np.ld}, src);
        o += nm;
      }
    }
    assign(P.P2M, np);
  }
  static void equalise(Blk& L, Blk& Pt) {  // the "_modified" truncations (F:1445-1460)
    if (L.c < Pt.c) Pt.c = L.c; else L.c = Pt.c;
  }
  Blk persist_copy(const Blk& src, int r, int c) {  // leading r x c block into a fresh allocation
    Blk t = newblk(r, c);
    copy(t, Blk{src.p, r, c, src.ld});
    return t;
  }
  Blk persist_adj(const Blk& src) {
    Blk t = newblk(src.c, src.r);
    geam(t, src, 1, C1, C0);
    return t;
  }

  void compress_P2P_Two_Ways(int j, int k, int b) {  // F:1424-1490
    ++st_compress;
    CompressOut kb, bk;
    compress_P2P_pair(j, k, b, kb, bk);
    Blk nLk = kb.nL, nPtb = kb.nPt, nLb = bk.nL, nPtk = bk.nPt;
    equalise(nLk, nPtk);
    equalise(nLb, nPtb);
    Box& K = T[j][k];
    Box& Bb = T[j][b];
    // The two halves (k's locals with b's multipoles; b's locals with k's
    // multipoles) touch disjoint blocks -- M2L[k][x] and M2L[x][b] against M2L[b][x]
    // and M2L[x][k], and the distinct parents of two well-separated boxes -- so
    // each stage of both halves is one batched launch.
    // stage 1: the new M2L blocks, the transfer matrices, the new bases
    Blk m2l_kb = persist_copy(kb.M2L, nLk.c, nPtb.c), m2l_bk = persist_copy(bk.M2L, nLb.c, nPtk.c);
    Blk Tk = scr(nLk.c, K.L2P.c), Tb = scr(Bb.P2M.r, nPtb.c);
    Blk Tk2 = scr(nLb.c, Bb.L2P.c), Tb2 = scr(K.P2M.r, nPtk.c);
    gemm(Tk, nLk, 1, K.L2P, 0, C1, C0);
    gemm(Tb, Bb.P2M, 0, nPtb, 0, C1, C0);
    gemm(Tk2, nLb, 1, Bb.L2P, 0, C1, C0);
    gemm(Tb2, K.P2M, 0, nPtk, 0, C1, C0);
    Blk Lk = persist_copy(nLk, nLk.r, nLk.c), Pmb = persist_adj(nPtb);
    Blk Lb = persist_copy(nLb, nLb.r, nLb.c), Pmk = persist_adj(nPtk);
    flush_geam();
    flush_gemm();
    // stage 2: the other M2L blocks of the four changed bases, and the parents
    assign(K.M2L[b], m2l_kb);
    update_other_M2Ls_at_k(j, k, b, Tk);
    update_other_M2Ls_at_b(j, k, b, Tb);
    if (j > 2) { update_parent_L2P(j, k, Tk); update_parent_P2M(j, b, Tb); }
    assign(K.L2P, Lk);
    assign(Bb.P2M, Pmb);
    K.NumL = K.L2P.c;
    Bb.NumM = Bb.P2M.r;
    assign(Bb.M2L[k], m2l_bk);
    update_other_M2Ls_at_k(j, b, k, Tk2);
    update_other_M2Ls_at_b(j, b, k, Tb2);
    if (j > 2) { update_parent_L2P(j, b, Tk2); update_parent_P2M(j, k, Tb2); }
    assign(Bb.L2P, Lb);
    assign(K.P2M, Pmk);
    Bb.NumL = Bb.L2P.c;
    K.NumM = K.P2M.r;
    flush_geam();
    flush_gemm();
    // the Q blocks were fresh pool allocations; return them
    drop(kb.nL); drop(kb.nPt); drop(bk.nL); drop(bk.nPt);
  }


  void compress_M2P_P2L(int j, int k, int b) {  // F:1492-1530 (k not eliminated, b eliminated)
    ++st_compress;
    Box& K = T[j][k];
    Box& Bb = T[j][b];
    // compress_M2P(j, k, b) (F:1561-1575) and compress_P2L(j, b, k) (F:1577-1591) in lockstep
    const Blk& Mkb = K.M2P[b];
    const Blk& Lbk = Bb.P2L[k];
    if (Mkb.r != K.L2P.r) throw Fail(AIFMM_ERR_NUMERIC, "compress_M2P: block rows mismatch");
    if (Lbk.c != K.P2M.c) throw Fail(AIFMM_ERR_NUMERIC, "compress_P2L: block cols mismatch");
    Blk Acol = scr(K.L2P.r, K.L2P.c + Mkb.c);
    copy(Blk{Acol.p, K.L2P.r, K.L2P.c, Acol.ld}, K.L2P);
    copy(Blk{Acol.p + (size_t)K.L2P.c * Acol.ld, Mkb.r, Mkb.c, Acol.ld}, Mkb);
    const int mk = K.P2M.c, rk = K.P2M.r;
    Blk Arow = scr(mk, rk + Lbk.r);
    geam(Blk{Arow.p, mk, rk, Arow.ld}, K.P2M, 1, C1, C0);
    geam(Blk{Arow.p + (size_t)rk * Arow.ld, mk, Lbk.r, Arow.ld}, Lbk, 1, C1, C0);
    flush_geam();
    QRF qc, qw;
    qr_prepare(qc, Acol, tol_factor, false);
    qr_prepare(qw, Arow, tol_factor, false);
    flush_qr();
    sync();
    int ic[2], iw[2];
    d2h(ic, qc.info, sizeof ic);
    d2h(iw, qw.info, sizeof iw);
    const int rc = ic[1], rr = iw[1];
    Blk nLk = newblk(Acol.r, rc), nPtk = newblk(Arow.r, rr);
    formq(qc, nLk);
    formq(qw, nPtk);
    flush_formq();
    Blk Rkp = scr(rc, Mkb.c), Rk = scr(rc, K.L2P.c), Rn = scr(rr, rk), Rnp = scr(rr, Lbk.r);
    gemm(Rkp, nLk, 1, Mkb, 0, C1, C0);
    gemm(Rk, nLk, 1, K.L2P, 0, C1, C0);
    gemm(Rn, nPtk, 1, K.P2M, 1, C1, C0);
    gemm(Rnp, nPtk, 1, Lbk, 1, C1, C0);
    flush_gemm();
    const Blk& m_kb = K.M2L[b];
    const Blk& m_bk = Bb.M2L[k];
    if (m_kb.r != K.L2P.c || m_bk.c != K.P2M.r) throw Fail(AIFMM_ERR_NUMERIC, "compress_M2P_P2L: M2L shape");
    Blk M2Lkb = scr(rc, m_kb.c), M2Lbk = scr(m_bk.r, rr);
    gemm(M2Lkb, Rk, 0, m_kb, 0, C1, C0);   // Rk M2L[k][b] + Rk'
    gemm(M2Lbk, m_bk, 0, Rn, 1, C1, C0);   // M2L[b][k] Rn^H + Rn'^H
    flush_gemm();
    geam(M2Lkb, Rkp, 0, C1, C1);
    geam(M2Lbk, Rnp, 1, C1, C1);
    flush_geam();
    equalise(nLk, nPtk);
    // k's locals and k's multipoles change; the updates touch M2L[k][x], M2L[x][k]
    // and two different blocks of k's parent, so each stage is one batched launch
    Blk m2l_kb = persist_copy(M2Lkb, nLk.c, M2Lkb.c), m2l_bk = persist_copy(M2Lbk, M2Lbk.r, nPtk.c);
    Blk Tk = scr(nLk.c, K.L2P.c), Tb = scr(K.P2M.r, nPtk.c);
    gemm(Tk, nLk, 1, K.L2P, 0, C1, C0);
    gemm(Tb, K.P2M, 0, nPtk, 0, C1, C0);
    Blk L = persist_copy(nLk, nLk.r, nLk.c), Pm = persist_adj(nPtk);
    flush_geam();
    flush_gemm();
    assign(K.M2L[b], m2l_kb);
    update_other_M2Ls_at_k(j, k, b, Tk);
    if (j > 2) update_parent_L2P(j, k, Tk);
    assign(Bb.M2L[k], m2l_bk);
    update_other_M2Ls_at_b(j, b, k, Tb);
    if (j > 2) update_parent_P2M(j, k, Tb);
    assign(K.L2P, L);
    assign(K.P2M, Pm);
    K.NumL = K.L2P.c;
    K.NumM = K.P2M.r;
    flush_geam();
    flush_gemm();
    drop(nLk);
    drop(nPtk);
  }

  void initialise_P2P_NonLeafLevel(int j) {  // F:1743-1807
    for (int k = 0; k < nBoxes[j]; ++k) {
      Box& B = T[j][k];
      auto mosaic = [&](int nn) {
        int nr = 0, nc = 0;
        for (int a = 0; a < 4; ++a) nr += T[j + 1][4 * k + a].NumL;
        for (int b = 0; b < 4; ++b) nc += T[j + 1][4 * nn + b].NumM;
        Blk P = newblk(nr, nc);
        int ri = 0;
        for (int a = 0; a < 4; ++a) {
          Box& ch = T[j + 1][4 * k + a];
          int ci = 0;
          for (int b = 0; b < 4; ++b) {
            const int cbx = 4 * nn + b, rr = ch.NumL, cc = T[j + 1][cbx].NumM;
            if (rr > 0 && cc > 0) {
              const Blk& src = ch.M2L[cbx];
              if (src.r != rr || src.c != cc)
                throw Fail(AIFMM_ERR_NUMERIC, "mosaic: child M2L block has the wrong shape");
              copy(Blk{P.p + ri + (size_t)ci * P.ld, rr, cc, P.ld}, src);
            } else if (rr > 0 && cc > 0) {
              // unreachable
            }
            ci += cc;
          }
          ri += ch.NumL;
        }
        return P;
      };
      for (int n = 0; n < 8; ++n) if (B.nb[n] != -1) { Blk P = mosaic(B.nb[n]); assign(B.P2P[B.nb[n]], P); }
      { Blk P = mosaic(k); assign(B.P2P[k], P); }
      if ((int)ged.size() > 20000) flush_geam();
    }
    flush_geam();
  }

  // The pairs queued by the previous box step (F:2411-2438): an instance is
  // queued when its fill-in norm exceeds 1e-10 at the time it was recorded, and
  // only instances involving k are compressed, in the order they were queued.
  // The x-phase norms are waited for first; a z-phase instance matters only if
  // its pair was not already queued by an x-phase instance (a repeated pair is
  // a no-op: its block is gone after the first compression), so the z-phase
  // norms (the end of the previous step's chain) are waited for only then.
  void take_pending(int j, int k, std::vector<std::pair<int, int>>& p2p, std::vector<std::pair<int, int>>& p2l) {
    p2p.clear(); p2l.clear();
    const int n = (int)cands.size();
    auto inv = [&](int i) { return cands[i].nn == k || cands[i].pp == k; };
    bool involved = false;
    for (int i = 0; i < n; ++i) if (inv(i)) { involved = true; break; }
    if (!involved) { clear_cands(); return; }
    const int nx = std::min(ncand[0], n);
    std::vector<char> take(n, 0);
    std::set<std::tuple<int, int, int>> queued;
    bool x_inv = false;
    for (int i = 0; i < nx; ++i) x_inv = x_inv || inv(i);
    if (x_inv) {
      wait_norms(0);
      for (int i = 0; i < nx; ++i)
        if (inv(i) && h_norms[i] > 1e-10) { take[i] = 1; queued.insert(std::make_tuple(cands[i].kind, cands[i].nn, cands[i].pp)); }
    }
    bool need_z = false;
    for (int i = nx; i < n; ++i)
      if (inv(i) && !queued.count(std::make_tuple(cands[i].kind, cands[i].nn, cands[i].pp))) { need_z = true; break; }
    if (need_z) {
      wait_norms(1);
      for (int i = nx; i < n; ++i)
        if (inv(i) && !queued.count(std::make_tuple(cands[i].kind, cands[i].nn, cands[i].pp)) && h_norms[i] > 1e-10)
          take[i] = 1;
    }
    for (int i = 0; i < n; ++i) {
      if (!take[i]) continue;
      if (cands[i].kind == 0) p2p.push_back({cands[i].nn, cands[i].pp});
      else p2l.push_back({cands[i].nn, cands[i].pp});
    }
    clear_cands();
    (void)j;
  }

  void eliminate_phase_efficient() {  // F:2407-2451
    std::vector<std::pair<int, int>> p2p, p2l;
    clear_cands();
    for (int j = depth; j >= 2; --j) {
      if (j != depth) initialise_P2P_NonLeafLevel(j);
      for (int k = 0; k < nBoxes[j]; ++k) {
        auto tp0 = std::chrono::steady_clock::now();
        eliminate_x_side(j, k);
        take_pending(j, k, p2p, p2l);
        for (auto& pr : p2p) {
          const int nn = pr.first, pp = pr.second;
          if (k != nn && k != pp) continue;
          if (T[j][nn].P2P[pp].size() != 0) {
            compress_P2P_Two_Ways(j, nn, pp);
            drop(T[j][nn].P2P[pp]);
            drop(T[j][pp].P2P[nn]);
          }
        }
        for (auto& pr : p2l) {
          const int nn = pr.first, pp = pr.second;
          if (k != nn && k != pp) continue;
          if (T[j][nn].P2L[pp].size() != 0) {
            compress_M2P_P2L(j, pp, nn);
            drop(T[j][nn].P2L[pp]);
            drop(T[j][pp].M2P[nn]);
          }
        }
        auto tp1 = std::chrono::steady_clock::now();
        T[j][k].elim = true;
        eliminate_x(j, k);
        eliminate_z(j, k);
        end_step();
        auto tp2 = std::chrono::steady_clock::now();
        st_pending_ms += std::chrono::duration<double, std::milli>(tp1 - tp0).count();
        st_elim_ms += std::chrono::duration<double, std::milli>(tp2 - tp1).count();
      }
      sync();
      clear_cands();  // pending pairs never cross a level
    }
    factor_base(2);
  }

  void end_step() {
    // scratch and deferred frees of this step can be reused once every kernel of
    // the step has been enqueued (single stream: later kernels run after them)
    scratch.reset();
    pool.commit_frees();
  }

  // F:2453-2485, factorisation half: the dense level-2 system (each box's
  // locals against every box's multipoles through the level's M2L blocks) is
  // factored once and kept for every solve.
  Blk base_A;
  QRF base_qr;
  int base_NL = 0, base_NM = 0;
  void factor_base(int j) {
    drop(base_A);
    drop_qrf(base_qr);
    int NM = 0, NL = 0;
    for (int k = 0; k < nBoxes[j]; ++k) { NM += T[j][k].NumM; NL += T[j][k].NumL; }
    base_NL = NL;
    base_NM = NM;
    if (NL == 0 || NM == 0) { end_step(); return; }
    base_A = newblk(NL, NM);
    zero(base_A);
    int ri = 0;
    for (int r = 0; r < nBoxes[j]; ++r) {
      Box& R = T[j][r];
      int si = 0;
      for (int s_ = 0; s_ < nBoxes[j]; ++s_) {
        const int nc = T[j][s_].NumM;
        if (R.NumL > 0 && nc > 0) {
          const Blk& m = R.M2L[s_];
          if (m.r != R.NumL || m.c != nc) throw Fail(AIFMM_ERR_NUMERIC, "base level: M2L block has the wrong shape");
          copy(Blk{base_A.p + ri + (size_t)si * base_A.ld, m.r, m.c, base_A.ld}, m);
        }
        si += nc;
      }
      ri += R.NumL;
    }
    flush_geam();
    qr_prepare(base_qr, base_A, 0.0, true);
    flush_qr();
    end_step();
  }

  // ---- solve with kept factors
  //
  // The reference carries the right-hand side through the elimination
  // (F:1968, 1997-2001, 2252, 2289-2293) and solves the base level (F:2453-2485)
  // and the back substitution (F:2487-2532) with it.  Eliminating box s
  // subtracts X[t][s] QRx_s^-1 r_s (eliminate_x) and L2P_f[t] y_s (eliminate_z)
  // from the right-hand side of every neighbour t: the particle one while t is
  // not eliminated (t > s), the multipole one after (t < s).  Every block in
  // these products is frozen once s is eliminated, except L2P_f, which the
  // elimination keeps per box and neighbour slot (Lf).  Gathered per receiving
  // box k, with rhs_k the leaf right-hand side or the children's multipole ones:
  //   sr_k  = rhs_k - sum_{nn < k} (P2P[k][nn] sxb_nn + Lf_{k,nn} sy_nn)
  //   sxb_k = QRx_k^-1 sr_k,  sy_k = QRz_k^-1 (-P2M_k sxb_k)
  //   smr_k = sy_k  - sum_{nn > k} (P2L[k][nn] sxb_nn + Lf_{k,nn} sy_nn)
  // where Lf_{k,nn} is the Lf of box nn at the slot that faces k.  sr_k needs
  // only smaller-index neighbours, so the forward sweep runs in waves like the
  // back substitution; smr needs the whole level and is one batch after it.
  std::vector<std::vector<std::vector<int>>> fwd_waves, bwd_waves;
  // wave(k) = 1 + the largest wave among k's neighbours that come before k in
  // the sweep (smaller index forward, larger index backward): the boxes of a
  // wave are pairwise non-adjacent and read only what earlier waves wrote.
  std::vector<std::vector<int>> level_waves(int j, bool forward) const {
    const int nbx = nBoxes[j];
    std::vector<int> wave(nbx, 0);
    int nw = 0;
    for (int t = 0; t < nbx; ++t) {
      const int k = forward ? t : nbx - 1 - t;
      int w = 0;
      for (int n = 0; n < 8; ++n) {
        const int nn = T[j][k].nb[n];
        if (nn != -1 && (forward ? nn < k : nn > k)) w = std::max(w, wave[nn] + 1);
      }
      wave[k] = w;
      nw = std::max(nw, w + 1);
    }
    std::vector<std::vector<int>> waves(nw);
    for (int t = 0; t < nbx; ++t) {
      const int k = forward ? t : nbx - 1 - t;
      waves[wave[k]].push_back(k);
    }
    return waves;
  }
  const Blk& lf_towards(int j, int k, int n) const {  // Lf of neighbour nb[n] at the slot facing k
    const Box& Nn = T[j][T[j][k].nb[n]];
    return Nn.Lf[(n + 4) & 7];
  }
  void forward_level(int j) {
    for (const auto& ks : fwd_waves[j]) {
      for (int k : ks) {
        Box& B = T[j][k];
        std::vector<std::pair<Blk, Blk>> terms;
        for (int n = 0; n < 8; ++n) {
          const int nn = B.nb[n];
          if (nn == -1 || nn > k) continue;
          terms.push_back({B.P2P[nn], T[j][nn].sxb});
          terms.push_back({lf_towards(j, k, n), T[j][nn].sy});
        }
        gemm_sum(B.sr, terms, CM1, C1);
      }
      flush_gemm();
      for (int k : ks) {
        Box& B = T[j][k];
        if (B.P2P[k].size() != 0) solve(B.qx, B.sr, B.sxb, C1);
      }
      flush_solve();
      std::vector<Blk> lr(ks.size());
      for (size_t q = 0; q < ks.size(); ++q) {
        Box& B = T[j][ks[q]];
        if (B.L2M_f.size() == 0) continue;
        lr[q] = scr(B.P2M.r, nrhs);
        gemm(lr[q], B.P2M, 0, B.sxb, 0, CM1, C0);
      }
      flush_gemm();
      for (size_t q = 0; q < ks.size(); ++q) {
        Box& B = T[j][ks[q]];
        if (B.L2M_f.size() != 0) solve(B.qz, lr[q], B.sy, C1);
      }
      flush_solve();
      end_step();
    }
    for (int k = 0; k < nBoxes[j]; ++k) copy(T[j][k].smr, T[j][k].sy);
    flush_geam();
    for (int k = 0; k < nBoxes[j]; ++k) {
      Box& B = T[j][k];
      std::vector<std::pair<Blk, Blk>> terms;
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1 || nn < k) continue;
        terms.push_back({B.P2L[nn], T[j][nn].sxb});
        terms.push_back({lf_towards(j, k, n), T[j][nn].sy});
      }
      gemm_sum(B.smr, terms, CM1, C1);
      if ((int)gd.size() > 20000) flush_gemm();
    }
    flush_gemm();
    end_step();
  }
  void solve_base_rhs(int j) {  // F:2453-2485, solve half
    if (base_NL == 0 || base_NM == 0) {
      for (int k = 0; k < nBoxes[j]; ++k) { Blk t = newblk(T[j][k].NumM, nrhs); zero(t); assign(T[j][k].multipoles, t); }
      return;
    }
    Blk b = scr(base_NL, nrhs);
    int ri = 0;
    for (int r = 0; r < nBoxes[j]; ++r) {
      Box& R = T[j][r];
      copy(Blk{b.p + ri, R.NumL, nrhs, b.ld}, R.smr);
      ri += R.NumL;
    }
    flush_geam();
    Blk mp = scr(base_NM, nrhs);
    solve(base_qr, b, mp, C1);
    flush_solve();
    int o = 0;
    for (int k = 0; k < nBoxes[j]; ++k) {
      Blk t = newblk(T[j][k].NumM, nrhs);
      copy(t, Blk{mp.p + o, T[j][k].NumM, nrhs, mp.ld});
      assign(T[j][k].multipoles, t);
      o += T[j][k].NumM;
    }
    flush_geam();
    end_step();
  }
  // F:2487-2532 (the factorisations of the elimination are reused).  The
  // reference visits the boxes of a level in decreasing order; box k reads the
  // particles of its neighbours with a larger index (already solved) and the
  // multipoles of the others (known from the level above).  The backward waves
  // give each box exactly what the sequential order gives it.
  // The particle right-hand side sr and the multipoles are updated in place: sr
  // is read by this box alone, and a box's multipoles only by its larger-index
  // neighbours, which earlier waves have finished (a parent's particles, which
  // hold its children's multipoles, are not read again either).
  void backward_wave(int j, const std::vector<int>& ks) {
    std::vector<Blk> t(ks.size());
    std::vector<int> act;  // boxes with unknowns at this level
    for (size_t q = 0; q < ks.size(); ++q)
      if (T[j][ks[q]].P2P[ks[q]].size() != 0) act.push_back((int)q);
    for (int q : act) {  // rhs1 = sr - sum of the neighbours' products
      const int k = ks[q];
      Box& B = T[j][k];
      std::vector<std::pair<Blk, Blk>> terms;
      for (int n = 0; n < 8; ++n) {
        const int nn = B.nb[n];
        if (nn == -1) continue;
        if (nn > k) terms.push_back({B.P2P[nn], T[j][nn].particles});
        else terms.push_back({B.M2P[nn], T[j][nn].multipoles});
      }
      gemm_sum(B.sr, terms, CM1, C1);
    }
    flush_gemm();
    for (int q : act) {  // t = QRx^-1 rhs1
      Box& B = T[j][ks[q]];
      t[q] = scr(B.P2P[ks[q]].c, nrhs);
      solve(B.qx, B.sr, t[q], C1);
    }
    flush_solve();
    for (int q : act) gemm(T[j][ks[q]].multipoles, T[j][ks[q]].P2M, 0, t[q], 0, CM1, C1);  // rhs2
    flush_gemm();
    for (int q : act) {  // locals = QRz^-1 rhs2
      Box& B = T[j][ks[q]];
      Blk loc = newblk(B.L2M_f.size() != 0 ? B.L2M_f.c : 0, nrhs);
      if (B.L2M_f.size() != 0) solve(B.qz, B.multipoles, loc, C1);
      assign(B.locals, loc);
    }
    flush_solve();
    for (int q : act) gemm(T[j][ks[q]].sr, T[j][ks[q]].L2P, 0, T[j][ks[q]].locals, 0, CM1, C1);  // v = rhs1 - L2P locals
    flush_gemm();
    for (int q : act) {  // particles = QRx^-1 v
      Box& B = T[j][ks[q]];
      Blk px = newblk(B.P2P[ks[q]].c, nrhs);
      solve(B.qx, B.sr, px, C1);
      assign(B.particles, px);
    }
    flush_solve();
    for (size_t q = 0; q < ks.size(); ++q) {
      const int k = ks[q];
      Box& B = T[j][k];
      if (B.P2P[k].size() == 0) { Blk px = newblk(0, nrhs); assign(B.particles, px); }
      if (j != depth) {
        int o = 0;
        for (int c = 0; c < 4; ++c) {
          Box& ch = T[j + 1][4 * k + c];
          Blk view{B.particles.p ? B.particles.p + o : nullptr, ch.NumM, nrhs, B.particles.ld, 0};
          ch.multipoles = view;  // a view: not owned
          o += ch.NumM;
        }
      }
    }
    end_step();
  }
  void release_solve_state() {
    for (auto& lv : T)
      for (auto& B : lv) {
        drop(B.sr); drop(B.sxb); drop(B.sy); drop(B.smr);
        drop(B.particles); drop(B.locals); drop(B.multipoles);
      }
  }

  void release_level_data() {
    for (auto& lv : T)
      for (auto& B : lv) {
        auto dm = [&](std::map<int, Blk>& m) { for (auto& kv : m) drop(kv.second); m.clear(); };
        dm(B.M2L); dm(B.P2P); dm(B.M2P); dm(B.P2L); dm(B.P2M_f); dm(B.M2M_f);
        for (auto& l : B.Lf) drop(l);
        drop(B.L2M_f);
        drop_qrf(B.qx); drop_qrf(B.qz);
        B.elim = false;
      }
    release_solve_state();
    release_plans();
    drop(base_A);
    drop_qrf(base_qr);
    factored = false;
  }
  // Everything a tree holds, before the tree is rebuilt: the elimination's blocks
  // and factorisations, the bases, the ACA factors and the kept copy of the
  // assembly.
  void release_tree() {
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(st2));
    if (have_saved) release_saved();
    have_saved = false;
    consumed = false;
    assembled = false;
    release_level_data();
    for (auto& lv : T)
      for (auto& B : lv) { drop(B.L2P); drop(B.P2M); drop(B.Ac); drop(B.Ar); }
    pool.commit_frees();
  }

  bool consumed = false;  // the elimination consumed the assembled blocks
  bool factored = false;  // factors are kept: solve() may run any number of times
  double ms_factor = 0, ms_solve = 0;
  long launches_factor = 0, launches_solve = 0;
  // eliminate_phase_efficient with the base-level factorisation (F:2407-2485),
  // right-hand side not carried
  // The mixed form factorises in complex64: its recompressions cannot resolve
  // ranks below this relative tolerance (a few units of FP32 rounding of a
  // 36-row block), so a tighter factor tolerance is raised to it.
  static constexpr double kC64MinTol = 1e-6;
  int factor_es = 16;
  void factorize(int flags, int precision = AIFMM_PRECISION_FP64) {
    if (!assembled) throw Fail(AIFMM_ERR_STATE, "assemble() must run before factorize()");
    if (consumed && !have_saved)
      throw Fail(AIFMM_ERR_STATE, "the assembly was consumed by a previous factorisation: assemble again, or pass AIFMM_KEEP_ASSEMBLY");
    auto t0 = std::chrono::steady_clock::now();
    const long l0 = launches_;
    release_plans();
    // the elimination consumes the assembled blocks; with AIFMM_KEEP_ASSEMBLY a
    // pristine copy is kept so that the handle can be factored again
    es_ = 16;  // the kept assembly is restored in complex128, then converted
    if ((flags & AIFMM_KEEP_ASSEMBLY) || have_saved) snapshot_restore();
    if (precision == AIFMM_PRECISION_C64) {
      es_ = 8;
      to_working_form();
    }
    release_solve_state();
    factored = false;
    consumed = true;
    factor_es = es_;
    const double tol_keep = tol_factor;
    if (es_ == 8) tol_factor = std::max(tol_factor, kC64MinTol);
    st_sync_ms = st_compress_ms = st_elim_ms = st_pending_ms = 0;
    st_syncs = st_compress = 0;
    try {
      eliminate_phase_efficient();
    } catch (...) {
      tol_factor = tol_keep;
      throw;
    }
    tol_factor = tol_keep;
    fwd_waves.assign(depth + 1, {});
    bwd_waves.assign(depth + 1, {});
    for (int j = 2; j <= depth; ++j) {
      fwd_waves[j] = level_waves(j, true);
      bwd_waves[j] = level_waves(j, false);
      for (int k = 0; k < nBoxes[j]; ++k)
        for (int n = 0; n < 8; ++n) {
          const int nn = T[j][k].nb[n];
          if (nn != -1 && T[j][nn].nb[(n + 4) & 7] != k) throw Fail(AIFMM_ERR_NUMERIC, "neighbour slots not mirrored");
        }
    }
    sync();
    CK(cudaStreamSynchronize(st2));
    prof_collect();
    pool.commit_frees();
    factored = true;
    launches_factor = launches_ - l0;
    ms_factor = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  // b and x: N x nrhs complex, column stride ldb / ldx (>= N), host or device.
  // With AIFMM_SOLVE_GRAPH the solve replays the CUDA graph of this right-hand-side
  // count (recorded by the first such solve after a factorisation).
  void solve_rhs(int nrhs_, const double* b, long ldb, double* x, long ldx, int flags) {
    if (!factored) throw Fail(AIFMM_ERR_STATE, "factorize() must run before solve()");
    if (nrhs_ < 1) throw Fail(AIFMM_ERR_ARG, "nrhs must be positive");
    if (ldb < N || ldx < N) throw Fail(AIFMM_ERR_ARG, "leading dimension smaller than the number of unknowns");
    auto t0 = std::chrono::steady_clock::now();
    const long l0 = launches_;
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const cudaMemcpyKind h2d = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind d2h_ = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (flags & AIFMM_SOLVE_GRAPH) {
      SolvePlan& pl = plan_for(nrhs_);
      CK(cudaMemcpy2DAsync(pl.bin, sizeof(double2) * N, b, sizeof(double2) * ldb, sizeof(double2) * N, nrhs_, h2d, st));
      CK(cudaGraphLaunch(pl.exec, st));
      CK(cudaMemcpy2DAsync(x, sizeof(double2) * ldx, pl.xout, sizeof(double2) * N, sizeof(double2) * N, nrhs_, d2h_, st));
      sync();
      launches_ += pl.launches;
    } else {
      const size_t bytes = sizeof(double2) * (size_t)N * nrhs_;
      Tmp tb(this, dev ? 1 : bytes), tx(this, dev ? 1 : bytes);
      const double2* db = reinterpret_cast<const double2*>(b);
      double2* dx = reinterpret_cast<double2*>(x);
      long lb = ldb, lx = ldx;
      if (!dev) {
        CK(cudaMemcpy2DAsync(tb.ptr, sizeof(double2) * N, b, sizeof(double2) * ldb, sizeof(double2) * N, nrhs_,
                             cudaMemcpyHostToDevice, st));
        db = tb.as<double2>();
        dx = tx.as<double2>();
        lb = lx = N;
      }
      solve_core(nrhs_, db, lb, dx, lx);
      if (!dev)
        CK(cudaMemcpy2DAsync(x, sizeof(double2) * ldx, dx, sizeof(double2) * N, sizeof(double2) * N, nrhs_,
                             cudaMemcpyDeviceToHost, st));
      sync();
      release_solve_state();
    }
    prof_collect();
    pool.commit_frees();
    launches_solve = launches_ - l0;
    ms_solve = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  // The solve on device buffers (the per-solve blocks stay in the boxes until
  // release_solve_state or a plan takes them).
  void solve_core(int nrhs_, const double2* db, long ldd_b, double2* dx, long ldd_x) {
    nrhs = nrhs_;
    cur = st;
    release_solve_state();
    for (int j = 2; j <= depth; ++j)
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& B = T[j][k];
        const int m = B.P2P[k].r;
        B.sr = newblk(m, nrhs);
        B.sxb = newblk(B.P2P[k].size() != 0 ? B.P2P[k].c : 0, nrhs);
        B.sy = newblk(B.L2M_f.size() != 0 ? B.L2M_f.c : 0, nrhs);
        B.smr = newblk(B.sy.r, nrhs);
      }
    // assign_Leaf_rhs (F:1092-1103)
    for (int k = 0; k < nBoxes[depth]; ++k) {
      Box& B = T[depth][k];
      copy(B.sr, Blk{const_cast<double2*>(db) + (size_t)k * rank, rank, nrhs, (int)ldd_b});
      if ((int)ged.size() > 20000) flush_geam();
    }
    flush_geam();
    for (int j = depth; j >= 2; --j) {
      if (j != depth) {  // the children's multipole right-hand sides (F:1798-1807)
        for (int k = 0; k < nBoxes[j]; ++k) {
          Box& B = T[j][k];
          int o = 0;
          for (int c = 0; c < 4; ++c) {
            const Blk& m = T[j + 1][4 * k + c].smr;
            copy(Blk{B.sr.p + o, m.r, nrhs, B.sr.ld}, m);
            o += m.r;
          }
          if (o != B.sr.r) throw Fail(AIFMM_ERR_NUMERIC, "children's multipole right-hand sides do not fill the parent's");
          if ((int)ged.size() > 20000) flush_geam();
        }
        flush_geam();
      }
      forward_level(j);
    }
    solve_base_rhs(2);
    for (int j = 2; j <= depth; ++j)
      for (const auto& ks : bwd_waves[j]) backward_wave(j, ks);
    // gather the leaf particles
    for (int k = 0; k < nBoxes[depth]; ++k) {
      const Blk& px = T[depth][k].particles;
      Blk dst{dx + (size_t)k * rank, rank, nrhs, (int)ldd_x};
      if (px.r == rank) copy(dst, px);
      else zero(dst);
      if ((int)ged.size() > 20000) flush_geam();
    }
    flush_geam();
  }

  // ---- autotuner: the GEMM tile width per product shape, from timings of both
  // widths on batches shaped like this problem's products (leaf blocks rank x rank,
  // their products with 8 right-hand sides, and the 4-rank blocks of the level
  // above), CUDA events on the handle's stream; the faster width is kept per shape.
  double tune_ms[2][2] = {{0, 0}, {0, 0}};  // [thin, wide][16, 32]
  void autotune() {
    const int r = rank, R = std::min(4 * rank, 160);
    const int nb = std::max(256, std::min(4096, nleaf / 2));  // the tree need not be built yet
    struct Shape { int m, n, k; };
    const Shape thin[2] = {{r, 8, r}, {R, 8, R}}, wide[2] = {{r, r, r}, {R, R, R}};
    size_t elems = 0;
    for (const Shape* sh : {thin, wide})
      for (int q = 0; q < 2; ++q) elems = std::max(elems, (size_t)sh[q].m * sh[q].k + (size_t)sh[q].k * sh[q].n +
                                                              (size_t)sh[q].m * sh[q].n);
    Tmp buf(this, sizeof(double2) * elems * nb);
    CK(cudaMemsetAsync(buf.ptr, 0, sizeof(double2) * elems * nb, st));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int bucket = 0; bucket < 2; ++bucket) {
      const Shape* sh = bucket == 0 ? thin : wide;
      for (int v = 0; v < 2; ++v) {
        gemm_cols[bucket] = v == 0 ? 16 : 32;
        float best = 1e30f;
        for (int rep_ = 0; rep_ < 6; ++rep_) {
          for (int j = 0; j < nb; ++j) {
            const Shape& z = sh[j & 1];
            double2* base = buf.as<double2>() + elems * j;
            Blk A{base, z.m, z.k, z.m}, B{base + (size_t)z.m * z.k, z.k, z.n, z.k};
            Blk C{base + (size_t)z.m * z.k + (size_t)z.k * z.n, z.m, z.n, z.m};
            gemm(C, A, 0, B, 0, C1, C1);
          }
          cur = st;
          CK(cudaEventRecord(e0, st));
          flush_gemm();
          CK(cudaEventRecord(e1, st));
          CK(cudaEventSynchronize(e1));
          float ms_ = 0.f;
          CK(cudaEventElapsedTime(&ms_, e0, e1));
          if (rep_ > 0) best = std::min(best, ms_);  // the first run warms up
        }
        tune_ms[bucket][v] = best;
      }
      gemm_cols[bucket] = tune_ms[bucket][0] < tune_ms[bucket][1] ? 16 : 32;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    sync();
    pool.commit_frees();
  }

  // ---- CUDA-graph plans: one per right-hand-side count, valid while the factors are
  struct SolvePlan {
    int nrhs = 0;
    double2* bin = nullptr;   // N x nrhs
    double2* xout = nullptr;  // N x nrhs
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<std::pair<void*, size_t>> owned;  // pool blocks: descriptors, per-solve state, bin, xout
    long launches = 0;
  };
  std::map<int, SolvePlan> plans;
  void release_plans() {
    for (auto& kv : plans) {
      SolvePlan& pl = kv.second;
      if (pl.exec) cudaGraphExecDestroy(pl.exec);
      if (pl.graph) cudaGraphDestroy(pl.graph);
      for (auto& o : pl.owned) pool.defer_free(o.first, o.second);
    }
    plans.clear();
  }
  SolvePlan& plan_for(int nr) {
    auto it = plans.find(nr);
    if (it != plans.end()) return it->second;
    SolvePlan pl;
    pl.nrhs = nr;
    const size_t vb = sizeof(double2) * (size_t)N * nr;
    pl.bin = static_cast<double2*>(pool.alloc(vb));
    pl.xout = static_cast<double2*>(pool.alloc(vb));
    pl.owned.push_back({pl.bin, vb});
    pl.owned.push_back({pl.xout, vb});
    CK(cudaMemsetAsync(pl.bin, 0, vb, st));
    // record: one eager solve whose descriptors go to plan-owned device blocks
    rec_ops.clear();
    rec_dev.clear();
    rec_host.clear();
    recording = true;
    const long l0 = launches_;
    try {
      solve_core(nr, pl.bin, N, pl.xout, N);
    } catch (...) {
      recording = false;
      throw;
    }
    recording = false;
    sync();
    rec_host.clear();
    pl.launches = launches_ - l0;
    for (auto& d : rec_dev) pl.owned.push_back(d);
    rec_dev.clear();
    // the per-solve blocks now belong to the plan (its graph addresses them)
    for (auto& lv : T)
      for (auto& B : lv) {
        for (Blk* b : {&B.sr, &B.sxb, &B.sy, &B.smr, &B.particles, &B.locals, &B.multipoles}) {
          if (b->p && b->cap) pl.owned.push_back({b->p.v(), b->cap});
          *b = Blk();
        }
      }
    // capture the recorded launches into a graph
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int err = 0;
    for (auto& op : rec_ops)
      if ((err = op(st)) != 0) break;
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    rec_ops.clear();
    if (err != 0 || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      for (auto& o : pl.owned) pool.defer_free(o.first, o.second);
      throw Fail(AIFMM_ERR_CUDA, std::string("solve graph capture failed: ") +
                                     cudaGetErrorString(err ? (cudaError_t)err : ce));
    }
    pl.graph = g;
    const cudaError_t ie = cudaGraphInstantiate(&pl.exec, g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      for (auto& o : pl.owned) pool.defer_free(o.first, o.second);
      throw Fail(AIFMM_ERR_CUDA, std::string("solve graph instantiation failed: ") + cudaGetErrorString(ie));
    }
    return plans.emplace(nr, std::move(pl)).first->second;
  }

  void factorize_solve(int nrhs_, const double* b, double* x, int flags) {
    if (nrhs_ < 1) throw Fail(AIFMM_ERR_ARG, "nrhs must be positive");
    auto t0 = std::chrono::steady_clock::now();
    factorize(flags);
    solve_rhs(nrhs_, b, N, x, N, flags);
    st_back_ms = ms_solve;
    launches_fs = launches_factor + launches_solve;
    ms[3] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  // ---- compressed matvec: y = A_c x with the kept pre-elimination assembly
  //
  // A_c is the matrix the assembly represents (the reference builds no such
  // product; it is the operator whose blocks FMM2DTree_find_error.hpp:1105-1361
  // and 1729-1741 assemble): the leaf near field P2P[k][nn] for the nine
  // neighbours (self included) plus, at every level j, the interaction-list
  // blocks L2P-chain M2L[k][kIL] P2M-chain.  With nested bases this is the H^2
  // product: multipoles upward (leaf P2M x, then P2M of the concatenated
  // children's multipoles), M2L at every level, locals downward (a parent's
  // L2P times its locals adds to its children's locals, which are consecutive
  // in Morton order), then L2P at the leaves plus the near field.
  void compressed_matvec(const double2* x, long ldx, double2* y, long ldy, int nr) {
    if (!have_saved) throw Fail(AIFMM_ERR_STATE, "the compressed product needs the kept assembly (AIFMM_KEEP_ASSEMBLY)");
    std::vector<std::vector<int>> mo(depth + 1), lo(depth + 1);
    std::vector<Blk> Mv(depth + 1), Lv(depth + 1);
    for (int j = 2; j <= depth; ++j) {
      int mt = 0, lt = 0;
      mo[j].resize(nBoxes[j] + 1);
      lo[j].resize(nBoxes[j] + 1);
      for (int k = 0; k < nBoxes[j]; ++k) {
        mo[j][k] = mt; mt += saved[j][k].NumM;
        lo[j][k] = lt; lt += saved[j][k].NumL;
      }
      mo[j][nBoxes[j]] = mt;
      lo[j][nBoxes[j]] = lt;
      Mv[j] = scr(mt, nr, 16);
      Lv[j] = scr(lt, nr, 16);
    }
    auto rows = [&](const Blk& v, int r0, int r1) { return Blk{v.p ? v.p + r0 : nullptr, r1 - r0, nr, v.ld}; };
    // upward: multipoles
    for (int k = 0; k < nBoxes[depth]; ++k) {
      const Saved& S = saved[depth][k];
      gemm(rows(Mv[depth], mo[depth][k], mo[depth][k + 1]), S.P2M, 0,
           Blk{const_cast<double2*>(x) + (size_t)k * rank, rank, nr, (int)ldx}, 0, C1, C0);
    }
    flush_gemm();
    for (int j = depth - 1; j >= 2; --j) {
      for (int k = 0; k < nBoxes[j]; ++k)
        gemm(rows(Mv[j], mo[j][k], mo[j][k + 1]), saved[j][k].P2M, 0,
             rows(Mv[j + 1], mo[j + 1][4 * k], mo[j + 1][4 * k + 4]), 0, C1, C0);
      flush_gemm();
    }
    // interaction lists: locals
    for (int j = 2; j <= depth; ++j) {
      for (int k = 0; k < nBoxes[j]; ++k) {
        const Box& B = T[j][k];
        std::vector<std::pair<Blk, Blk>> terms;
        auto add = [&](int kIL) {
          auto it = saved[j][k].M2L.find(kIL);
          if (it == saved[j][k].M2L.end()) return;
          terms.push_back({it->second, rows(Mv[j], mo[j][kIL], mo[j][kIL + 1])});
        };
        for (int i = 0; i < 16; ++i) if (B.inner[i] != -1) add(B.inner[i]);
        for (int i = 0; i < 24; ++i) if (B.outer[i] != -1) add(B.outer[i]);
        gemm_sum(rows(Lv[j], lo[j][k], lo[j][k + 1]), terms, C1, C0);
        if ((int)gd.size() > 20000) flush_gemm();
      }
      flush_gemm();
    }
    // downward: a parent's L2P times its locals adds to its children's locals
    for (int j = 2; j < depth; ++j) {
      for (int k = 0; k < nBoxes[j]; ++k)
        gemm(rows(Lv[j + 1], lo[j + 1][4 * k], lo[j + 1][4 * k + 4]), saved[j][k].L2P, 0,
             rows(Lv[j], lo[j][k], lo[j][k + 1]), 0, C1, C1);
      flush_gemm();
    }
    // leaves: near field plus L2P times the locals
    for (int k = 0; k < nBoxes[depth]; ++k) {
      const Box& B = T[depth][k];
      const Saved& S = saved[depth][k];
      std::vector<std::pair<Blk, Blk>> terms;
      auto near = [&](int nn) {
        auto it = S.P2P.find(nn);
        if (it == S.P2P.end()) throw Fail(AIFMM_ERR_NUMERIC, "kept assembly lacks a leaf near-field block");
        terms.push_back({it->second, Blk{const_cast<double2*>(x) + (size_t)nn * rank, rank, nr, (int)ldx}});
      };
      for (int n = 0; n < 8; ++n) if (B.nb[n] != -1) near(B.nb[n]);
      near(k);
      terms.push_back({S.L2P, rows(Lv[depth], lo[depth][k], lo[depth][k + 1])});
      gemm_sum(Blk{y + (size_t)k * rank, rank, nr, (int)ldy}, terms, C1, C0);
      if ((int)gd.size() > 20000) flush_gemm();
    }
    flush_gemm();
    end_step();
  }

  // ---- GMRES refinement against the compressed product
  //
  // Right-preconditioned restarted GMRES on A_c x = b with the kept
  // factorisation as the preconditioner M^-1 (solve_rhs), all in FP64: the
  // factors may come from a looser recompression tolerance than the assembly
  // (aifmm_set_factor_tolerance), the residual is always the assembly's.  The
  // nrhs columns run as independent Krylov processes in lockstep; the
  // Hessenberg matrices and Givens rotations live on the host.
  int gm_iters = 0;
  double gm_relres = 0;
  void refine_solve(int nr, const double* b, long ldb, double* x, long ldx, int flags, double rtol, int maxit,
                    int restart) {
    if (!factored) throw Fail(AIFMM_ERR_STATE, "factorize() must run before a refined solve");
    if (!have_saved) throw Fail(AIFMM_ERR_STATE, "a refined solve needs the kept assembly (factorize with AIFMM_KEEP_ASSEMBLY)");
    if (nr < 1 || restart < 1 || maxit < 0 || !(rtol > 0)) throw Fail(AIFMM_ERR_ARG, "invalid refinement parameters");
    if (ldb < N || ldx < N) throw Fail(AIFMM_ERR_ARG, "leading dimension smaller than the number of unknowns");
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const size_t vb = sizeof(double2) * (size_t)N * nr;
    const int m = restart;
    Tmp tB(this, vb), tX(this, vb), tW(this, vb), tZ(this, vb), tV(this, vb * (m + 1));
    Tmp tc(this, sizeof(double2) * nr * 2);
    double2* B = tB.as<double2>();
    double2* X = tX.as<double2>();
    double2* W = tW.as<double2>();
    double2* Z = tZ.as<double2>();
    double2* V = tV.as<double2>();
    double2* dcoef = tc.as<double2>();
    auto Vi = [&](int i) { return V + (size_t)i * N * nr; };
    if (dev) CK(cudaMemcpy2DAsync(B, sizeof(double2) * N, b, sizeof(double2) * ldb, sizeof(double2) * N, nr,
                                  cudaMemcpyDeviceToDevice, st));
    else CK(cudaMemcpy2DAsync(B, sizeof(double2) * N, b, sizeof(double2) * ldb, sizeof(double2) * N, nr,
                              cudaMemcpyHostToDevice, st));
    auto dots = [&](const double2* a, const double2* c, std::vector<double2>& out) {
      int e = aifmm_launch_coldot(a, N, c, N, N, nr, dcoef, st);
      if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
      out.resize(nr);
      d2h(out.data(), dcoef, sizeof(double2) * nr);
    };
    // y(:,c) = alpha_c x(:,c) + beta_c y(:,c)
    auto axpby = [&](const double2* xx, double2* yy, const std::vector<double2>& al, const std::vector<double2>& be) {
      std::vector<double2> ab(2 * nr);
      for (int c = 0; c < nr; ++c) { ab[c] = al[c]; ab[nr + c] = be[c]; }
      const double2* dab = static_cast<const double2*>(stage.put_raw(ab.data(), sizeof(double2) * 2 * nr, st));
      int e = aifmm_launch_colaxpby(xx, N, yy, N, N, nr, dab, dab + nr, st);
      if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    };
    auto precond = [&](const double2* in, double2* out) {  // out = M^-1 in, one graph per nrhs
      solve_rhs(nr, reinterpret_cast<const double*>(in), N, reinterpret_cast<double*>(out), N,
                AIFMM_PTR_DEVICE | AIFMM_SOLVE_GRAPH);
    };
    const std::vector<double2> one(nr, C1), mone(nr, CM1), zero_(nr, C0);
    std::vector<double2> d;
    dots(B, B, d);
    std::vector<double> bn(nr);
    for (int c = 0; c < nr; ++c) bn[c] = std::sqrt(d[c].x) > 0 ? std::sqrt(d[c].x) : 1.0;
    precond(B, X);  // the direct solve is the starting guess
    int it = 0, cycle = 0;
    double worst = 0, worst_prev = 0;
    for (;; ++cycle) {
      // true residual r = b - A_c x into V_0
      compressed_matvec(X, N, W, N, nr);
      CK(cudaMemcpyAsync(Vi(0), B, vb, cudaMemcpyDeviceToDevice, st));
      axpby(W, Vi(0), mone, one);
      dots(Vi(0), Vi(0), d);
      std::vector<double> beta(nr);
      worst = 0;
      for (int c = 0; c < nr; ++c) { beta[c] = std::sqrt(d[c].x); worst = std::max(worst, beta[c] / bn[c]); }
      if (worst <= rtol || it >= maxit) break;
      // With complex64 factors, a cycle that does not halve the true residual means
      // the preconditioner is not the linear operator GMRES assumes (a deep tree:
      // the elimination's internal growth times FP32 rounding): stop rather than
      // iterate to maxit.
      if (factor_es == 8 && cycle > 0 && !(worst <= 0.5 * worst_prev)) {
        gm_iters = it;
        gm_relres = worst;
        throw Fail(AIFMM_ERR_NUMERIC, "GMRES refinement stagnates: relative residual " + std::to_string(worst) +
                                          " after " + std::to_string(it) + " iterations (the factors are not an "
                                          "effective preconditioner)");
      }
      worst_prev = worst;
      {
        std::vector<double2> sc(nr);
        for (int c = 0; c < nr; ++c) sc[c] = make_double2(beta[c] > 0 ? 1.0 / beta[c] : 0.0, 0.0);
        axpby(Vi(0), Vi(0), zero_, sc);
      }
      // per column: H (m+1) x m column-major, Givens (cs, sn), g
      std::vector<std::vector<double2>> H(nr, std::vector<double2>((size_t)(m + 1) * m, C0));
      std::vector<std::vector<double>> cs(nr, std::vector<double>(m));
      std::vector<std::vector<double2>> sn(nr, std::vector<double2>(m)), g(nr, std::vector<double2>(m + 1, C0));
      for (int c = 0; c < nr; ++c) g[c][0] = make_double2(beta[c], 0.0);
      // with complex64 factors the first cycle is short, so that a stagnating
      // refinement is noticed early
      const int mk = cycle == 0 && factor_es == 8 ? std::min(m, 10) : m;
      int k = 0;
      for (; k < mk && it < maxit; ++k, ++it) {
        precond(Vi(k), Z);
        compressed_matvec(Z, N, W, N, nr);
        for (int l = 0; l <= k; ++l) {  // modified Gram-Schmidt
          dots(Vi(l), W, d);
          std::vector<double2> neg(nr);
          for (int c = 0; c < nr; ++c) { H[c][l + (size_t)k * (m + 1)] = d[c]; neg[c] = make_double2(-d[c].x, -d[c].y); }
          axpby(Vi(l), W, neg, one);
        }
        dots(W, W, d);
        std::vector<double2> sc(nr);
        double est = 0;
        for (int c = 0; c < nr; ++c) {
          const double h1 = std::sqrt(d[c].x);
          H[c][k + 1 + (size_t)k * (m + 1)] = make_double2(h1, 0.0);
          sc[c] = make_double2(h1 > 1e-300 ? 1.0 / h1 : 0.0, 0.0);
          // apply the previous rotations to column k, then a new one that zeroes H(k+1, k)
          double2* hk = &H[c][(size_t)k * (m + 1)];
          for (int l = 0; l < k; ++l) {
            const double2 a = hk[l], bb = hk[l + 1];
            const double2 s_ = sn[c][l];
            // [c s; -conj(s) c] [a; b]
            hk[l] = make_double2(cs[c][l] * a.x + (s_.x * bb.x - s_.y * bb.y), cs[c][l] * a.y + (s_.x * bb.y + s_.y * bb.x));
            hk[l + 1] = make_double2(cs[c][l] * bb.x - (s_.x * a.x + s_.y * a.y), cs[c][l] * bb.y - (s_.x * a.y - s_.y * a.x));
          }
          const double2 a = hk[k], bb = hk[k + 1];
          const double na = std::hypot(a.x, a.y), nb = std::hypot(bb.x, bb.y);
          if (nb == 0.0) { cs[c][k] = 1.0; sn[c][k] = C0; }
          else if (na == 0.0) { cs[c][k] = 0.0; sn[c][k] = make_double2(bb.x / nb, -bb.y / nb); }
          else {
            const double r = std::hypot(na, nb);
            cs[c][k] = na / r;
            // s = (a / |a|) conj(b) / r
            const double2 u = make_double2(a.x / na, a.y / na);
            sn[c][k] = make_double2((u.x * bb.x + u.y * bb.y) / r, (u.y * bb.x - u.x * bb.y) / r);
          }
          const double2 a2 = hk[k];
          const double2 s_ = sn[c][k];
          hk[k] = make_double2(cs[c][k] * a2.x + (s_.x * bb.x - s_.y * bb.y), cs[c][k] * a2.y + (s_.x * bb.y + s_.y * bb.x));
          hk[k + 1] = C0;
          const double2 gk = g[c][k];
          g[c][k] = make_double2(cs[c][k] * gk.x, cs[c][k] * gk.y);
          g[c][k + 1] = make_double2(-(s_.x * gk.x + s_.y * gk.y), -(s_.x * gk.y - s_.y * gk.x));
          est = std::max(est, std::hypot(g[c][k + 1].x, g[c][k + 1].y) / bn[c]);
        }
        axpby(W, Vi(k + 1), sc, zero_);
        if (est <= rtol) { ++k; ++it; break; }
      }
      // y = R^-1 g (back substitution per column), u = V y, x += M^-1 u
      CK(cudaMemsetAsync(W, 0, vb, st));
      std::vector<std::vector<double2>> yv(nr, std::vector<double2>(k, C0));
      for (int c = 0; c < nr; ++c)
        for (int l = k - 1; l >= 0; --l) {
          double2 sum = g[c][l];
          for (int q = l + 1; q < k; ++q) sum = csub(sum, cmul(H[c][l + (size_t)q * (m + 1)], yv[c][q]));
          const double2 dd = H[c][l + (size_t)l * (m + 1)];
          yv[c][l] = (dd.x == 0.0 && dd.y == 0.0) ? C0 : cdiv(sum, dd);
        }
      for (int l = 0; l < k; ++l) {
        std::vector<double2> al(nr);
        for (int c = 0; c < nr; ++c) al[c] = yv[c][l];
        axpby(Vi(l), W, al, one);
      }
      precond(W, Z);
      axpby(Z, X, one, one);
    }
    gm_iters = it;
    gm_relres = worst;
    if (dev) CK(cudaMemcpy2DAsync(x, sizeof(double2) * ldx, X, sizeof(double2) * N, sizeof(double2) * N, nr,
                                  cudaMemcpyDeviceToDevice, st));
    else CK(cudaMemcpy2DAsync(x, sizeof(double2) * ldx, X, sizeof(double2) * N, sizeof(double2) * N, nr,
                              cudaMemcpyDeviceToHost, st));
    sync();
    pool.commit_frees();
  }

  // Saved copy of the assembled state (L2P, P2M, M2L, leaf P2P) so that
  // factorize_solve can run more than once on one assembly.
  struct Saved { Blk L2P, P2M; std::map<int, Blk> M2L, P2P; int NumM, NumL; };
  std::vector<std::vector<Saved>> saved;
  bool have_saved = false;
  void release_saved() {
    for (auto& lv : saved)
      for (auto& S : lv) {
        drop(S.L2P); drop(S.P2M);
        for (auto& kv : S.M2L) drop(kv.second);
        for (auto& kv : S.P2P) drop(kv.second);
      }
    saved.clear();
    pool.commit_frees();
  }
  // The live (to be eliminated) blocks in complex64 for the mixed form.  The
  // interpolative bases carry the contrast's dynamic range: a column of
  // L2P = A(rows, skel) D^-1 scales with 1 / q(skeleton point), up to about
  // 1 / tolerance in the far corners of a Gaussian contrast, which FP32 cannot
  // carry next to O(1) entries.  So the conversion first equilibrates the
  // compressed representation by a diagonal similarity transform of every box's
  // local and multipole spaces -- locals l = S l', multipoles m' = T m, with
  // S = diag(sigma), T = diag(tau) -- chosen bottom-up so that every L2P has unit
  // columns and every P2M unit rows:
  //   L2P' = S_children^-1 L2P S,  P2M' = T P2M T_children^-1,  M2L' = S_k^-1 M2L T_j^-1,
  // (no children factor at the leaves; the leaf particle space and the leaf P2P
  // blocks are unchanged, so right-hand sides and solutions need no scaling).
  void to_working_form() {
    if (es_ == 16) return;
    std::vector<std::vector<long>> loff(depth + 2), moff(depth + 2);
    long totL = 0, totM = 0;
    for (int j = 2; j <= depth; ++j) {
      loff[j].resize(nBoxes[j] + 1);
      moff[j].resize(nBoxes[j] + 1);
      for (int k = 0; k < nBoxes[j]; ++k) {
        loff[j][k] = totL; totL += T[j][k].NumL;
        moff[j][k] = totM; totM += T[j][k].NumM;
      }
      loff[j][nBoxes[j]] = totL;
      moff[j][nBoxes[j]] = totM;
    }
    Tmp tS(this, sizeof(double) * 2 * std::max(1L, totL)), tT(this, sizeof(double) * 2 * std::max(1L, totM));
    double* sig = tS.as<double>();
    double* isig = sig + std::max(1L, totL);
    double* tau = tT.as<double>();
    double* itau = tau + std::max(1L, totM);
    for (int j = depth; j >= 2; --j) {
      std::vector<EquilDesc> ed;
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& B = T[j][k];
        if (B.L2P.p.es != 16 || B.P2M.p.es != 16) throw Fail(AIFMM_ERR_STATE, "equilibration needs the complex128 bases");
        if (B.L2P.c != B.NumL || B.P2M.r != B.NumM) throw Fail(AIFMM_ERR_NUMERIC, "equilibration: basis shapes");
        if (j < depth && (B.L2P.r != loff[j + 1][4 * k + 4] - loff[j + 1][4 * k] ||
                          B.P2M.c != moff[j + 1][4 * k + 4] - moff[j + 1][4 * k]))
          throw Fail(AIFMM_ERR_NUMERIC, "equilibration: children's spaces");
        if (B.L2P.size()) {
          EquilDesc e; e.A = B.L2P.p.d(); e.lda = B.L2P.ld; e.m = B.L2P.r; e.n = B.L2P.c; e.mode = 0;
          e.scale = j < depth ? isig + loff[j + 1][4 * k] : nullptr;
          e.s = sig + loff[j][k]; e.is = isig + loff[j][k];
          ed.push_back(e);
        } else if (B.NumL > 0) {
          throw Fail(AIFMM_ERR_NUMERIC, "equilibration: empty L2P with locals");
        }
        if (B.P2M.size()) {
          EquilDesc e; e.A = B.P2M.p.d(); e.lda = B.P2M.ld; e.m = B.P2M.r; e.n = B.P2M.c; e.mode = 1;
          e.scale = j < depth ? itau + moff[j + 1][4 * k] : nullptr;
          e.s = tau + moff[j][k]; e.is = itau + moff[j][k];
          ed.push_back(e);
        } else if (B.NumM > 0) {
          throw Fail(AIFMM_ERR_NUMERIC, "equilibration: empty P2M with multipoles");
        }
      }
      if (!ed.empty()) {
        const EquilDesc* d = stage.put(ed, st);
        KL(aifmm_launch_equilibrate(d, (int)ed.size(), st));
      }
    }
    auto conv = [&](Blk& b, const double* rs, const double* cs) {
      if (b.size() == 0) { b.p.es = es_; return; }
      Blk t = newblk(b.r, b.c);
      GeamDesc g; g.A = b.p.v(); g.C = t.p.v(); g.lda = b.ld; g.ldc = t.ld; g.opA = 0; g.m = b.r; g.n = b.c;
      g.esA = b.p.es; g.esC = t.p.es; g.alpha = C1; g.beta = C0; g.rs = rs; g.cs = cs;
      ged.push_back(g);
      assign(b, t);
    };
    for (int j = 2; j <= depth; ++j)
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& B = T[j][k];
        conv(B.L2P, j < depth ? isig + loff[j + 1][4 * k] : nullptr, sig + loff[j][k]);
        conv(B.P2M, tau + moff[j][k], j < depth ? itau + moff[j + 1][4 * k] : nullptr);
        for (auto& kv : B.M2L) conv(kv.second, isig + loff[j][k], itau + moff[j][kv.first]);
        for (auto& kv : B.P2P) {
          if (j != depth && kv.second.size()) throw Fail(AIFMM_ERR_STATE, "non-leaf P2P before the elimination");
          conv(kv.second, nullptr, nullptr);
        }
        for (auto* m : {&B.M2P, &B.P2L, &B.P2M_f, &B.M2M_f})
          for (auto& kv : *m)
            if (kv.second.size()) throw Fail(AIFMM_ERR_STATE, "elimination blocks before the elimination");
        if ((int)ged.size() > 20000) flush_geam();
      }
    flush_geam();
  }
  void snapshot_restore() {
    if (!have_saved) {
      saved.assign(depth + 1, {});
      for (int j = 2; j <= depth; ++j) {
        saved[j].resize(nBoxes[j]);
        for (int k = 0; k < nBoxes[j]; ++k) {
          Box& B = T[j][k];
          Saved& S = saved[j][k];
          S.NumM = B.NumM; S.NumL = B.NumL;
          S.L2P = newblk(B.L2P.r, B.L2P.c, 16); copy(S.L2P, B.L2P);
          S.P2M = newblk(B.P2M.r, B.P2M.c, 16); copy(S.P2M, B.P2M);
          for (auto& kv : B.M2L) { Blk t = newblk(kv.second.r, kv.second.c, 16); copy(t, kv.second); S.M2L[kv.first] = t; }
          if (j == depth)
            for (auto& kv : B.P2P) {
              Blk t = newblk(kv.second.r, kv.second.c, 16);
              copy(t, kv.second);
              S.P2P[kv.first] = t;
            }
          if ((int)ged.size() > 20000) flush_geam();
        }
      }
      flush_geam();
      have_saved = true;
      return;  // the live state is still pristine
    }
    release_level_data();
    for (int j = 2; j <= depth; ++j)
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& B = T[j][k];
        Saved& S = saved[j][k];
        B.NumM = S.NumM; B.NumL = S.NumL;
        { Blk t = newblk(S.L2P.r, S.L2P.c); copy(t, S.L2P); assign(B.L2P, t); }
        { Blk t = newblk(S.P2M.r, S.P2M.c); copy(t, S.P2M); assign(B.P2M, t); }
        for (auto& kv : S.M2L) { Blk t = newblk(kv.second.r, kv.second.c); copy(t, kv.second); B.M2L[kv.first] = t; }
        for (auto& kv : S.P2P) { Blk t = newblk(kv.second.r, kv.second.c); copy(t, kv.second); B.P2P[kv.first] = t; }
        if ((int)ged.size() > 20000) flush_geam();
      }
    flush_geam();
    pool.commit_frees();
  }
};

// ============================================================================
// Leaf tables without allocation (aifmm_tables_compute_noalloc)
//
// Some callers cannot let a library call cudaMalloc: applications that reserve
// the GPU's memory up front and hand out every byte through their own
// allocator, and latency-sensitive loops for which the device synchronisation
// that cudaMalloc / cudaFree may imply is not acceptable.  For them the table
// quadrature has a variant whose scratch (far-field moments, near-field
// integrals, the pseudo-inverse, a status word) lives in one file-scope device
// array of kTablesScratchBytes.  Every GPU that loads this library holds that
// array until the process exits.
// ============================================================================
namespace {
constexpr size_t kTablesScratchBytes = size_t(1) << 20;  // 1 MiB
__device__ __align__(256) unsigned char g_tables_scratch[kTablesScratchBytes];
constexpr int kMaxDevices = 64;
std::atomic<void*> g_scratch_addr[kMaxDevices];
}  // namespace

extern "C" aifmm_status aifmm_tables_compute_noalloc(aifmm_problem* p, double* M_dev, double* near_dev) {
  if (!p || !M_dev || !near_dev) return AIFMM_ERR_ARG;
  if (p->device < 0 || p->device >= kMaxDevices) return AIFMM_ERR_ARG;
  if (cudaSetDevice(p->device) != cudaSuccess) return AIFMM_ERR_CUDA;
  // the symbol's device address, looked up once per device with that device
  // current (threads that race here all store the same address)
  void* base = g_scratch_addr[p->device].load(std::memory_order_acquire);
  if (!base) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_tables_scratch) != cudaSuccess || !ptr) return AIFMM_ERR_CUDA;
    g_scratch_addr[p->device].store(ptr, std::memory_order_release);
    base = ptr;
  }
  const int rank = p->rank, nb = p->nb;
  // scratch layout: C (121 x nb) | V (9 rank x nb) | Q^+ (nb x rank doubles) | status
  const size_t offC = 0;
  const size_t offV = (offC + sizeof(double2) * 121 * (size_t)nb + 255) & ~size_t(255);
  const size_t offQ = (offV + sizeof(double2) * 9 * (size_t)rank * nb + 255) & ~size_t(255);
  const size_t offS = (offQ + sizeof(double) * (size_t)nb * rank + 255) & ~size_t(255);
  if (offS + sizeof(int) > kTablesScratchBytes) return AIFMM_ERR_ARG;  // problem larger than the fixed scratch
  char* sc = static_cast<char*>(base);
  double2* Cw = reinterpret_cast<double2*>(sc + offC);
  double2* Vw = reinterpret_cast<double2*>(sc + offV);
  double* qp = reinterpret_cast<double*>(sc + offQ);
  int* status = reinterpret_cast<int*>(sc + offS);
  // small inputs from fixed-size host arrays through the handle's preallocated pinned ring
  double glx[10], glw[10];
  gauss_legendre10(glx, glw);
  int2 basis[64];
  int t = 0;
  for (int dd = 0; dd < p->d.degree; ++dd)
    for (int a = 0; a < dd + 1; ++a) basis[t++] = make_int2(a, dd - a);  // LS/FarFieldInteraction.hpp:46-54
  double cheb[16];
  const double PI = 3.1415926535897932384;
  for (int k = 0; k < p->d.n_cheb; ++k) cheb[k] = -std::cos((k + 0.5) / p->d.n_cheb * PI);
  double r = p->d.L;
  for (int j = 0; j < p->depth; ++j) r = r / 2.0;
  const double* dx;
  const double* dw;
  const int2* db;
  const double* dc;
  try {
    dx = static_cast<const double*>(p->stage.put_raw(glx, sizeof glx, p->st));
    dw = static_cast<const double*>(p->stage.put_raw(glw, sizeof glw, p->st));
    db = static_cast<const int2*>(p->stage.put_raw(basis, sizeof(int2) * nb, p->st));
    dc = static_cast<const double*>(p->stage.put_raw(cheb, sizeof(double) * p->d.n_cheb, p->st));
  } catch (...) {
    return AIFMM_ERR_CUDA;
  }
  // the array keeps the previous call's contents: the status word must start at zero
  if (cudaMemsetAsync(status, 0, sizeof(int), p->st) != cudaSuccess) return AIFMM_ERR_CUDA;
  if (aifmm_launch_tables(p->d.n_cheb, p->d.degree, p->d.kappa, r, dx, dw, db, dc, Cw, Vw, status, qp,
                          reinterpret_cast<double2*>(M_dev), reinterpret_cast<double2*>(near_dev), p->st) != 0)
    return AIFMM_ERR_CUDA;
  int h_status = 0;
  if (cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, p->st) != cudaSuccess) return AIFMM_ERR_CUDA;
  if (cudaStreamSynchronize(p->st) != cudaSuccess) return AIFMM_ERR_CUDA;
  return h_status ? AIFMM_ERR_NUMERIC : AIFMM_OK;
}

// ============================================================================
// C ABI
// ============================================================================
namespace {
template <class F>
aifmm_status guard(aifmm_problem* p, F&& f) {
  try {
    if (p) CK(cudaSetDevice(p->device));
    f();
    if (p) p->err.clear();
    return AIFMM_OK;
  } catch (const Fail& e) {
    if (p) p->err = e.what();
    return e.st;
  } catch (const std::exception& e) {
    if (p) p->err = e.what();
    return AIFMM_ERR_NUMERIC;
  }
}
}  // namespace

extern "C" {

const char* aifmm_status_string(aifmm_status s) {
  switch (s) {
    case AIFMM_OK: return "ok";
    case AIFMM_ERR_ARG: return "invalid argument";
    case AIFMM_ERR_CUDA: return "CUDA error";
    case AIFMM_ERR_STATE: return "call out of order";
    case AIFMM_ERR_NOMEM: return "out of device memory";
    case AIFMM_ERR_NUMERIC: return "numerical / shape error";
    case AIFMM_ERR_NODEVICE: return "no CUDA device";
  }
  return "unknown status";
}

aifmm_status aifmm_problem_create(const aifmm_desc* desc, int device, aifmm_problem** out) {
  if (!desc || !out) return AIFMM_ERR_ARG;
  *out = nullptr;
  aifmm_problem* p = new aifmm_problem();
  try {
    p->create(*desc, device);
  } catch (const Fail& e) {
    aifmm_status s = e.st;
    p->destroy();
    delete p;
    return s;
  }
  *out = p;
  return AIFMM_OK;
}

aifmm_status aifmm_problem_destroy(aifmm_problem* p) {
  if (!p) return AIFMM_ERR_ARG;
  cudaSetDevice(p->device);
  p->destroy();
  delete p;
  return AIFMM_OK;
}

const char* aifmm_last_error(const aifmm_problem* p) { return p ? p->err.c_str() : "null handle"; }

aifmm_status aifmm_tables_compute(aifmm_problem* p, int round6_) {
  if (!p) return AIFMM_ERR_ARG;
  return guard(p, [&] { p->tables_compute(round6_); });
}

aifmm_status aifmm_tables_set(aifmm_problem* p, const double* M, const double* near_tables) {
  if (!p || !M || !near_tables) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    CK(cudaMemcpyAsync(p->d_M, M, sizeof(double2) * 121 * p->rank, cudaMemcpyHostToDevice, p->st));
    CK(cudaMemcpyAsync(p->d_near, near_tables, sizeof(double2) * 9 * p->rank * p->rank, cudaMemcpyHostToDevice, p->st));
    p->sync();
    p->tables_ready = true;
  });
}

aifmm_status aifmm_tables_get(aifmm_problem* p, double* M, double* near_tables) {
  if (!p || !M || !near_tables) return AIFMM_ERR_ARG;
  if (!p->tables_ready) { p->err = "tables not ready"; return AIFMM_ERR_STATE; }
  return guard(p, [&] {
    p->sync();
    p->d2h(M, p->d_M, sizeof(double2) * 121 * p->rank);
    p->d2h(near_tables, p->d_near, sizeof(double2) * 9 * p->rank * p->rank);
  });
}

aifmm_status aifmm_num_points(const aifmm_problem* p, int* n) {
  if (!p || !n) return AIFMM_ERR_ARG;
  *n = p->N;
  return AIFMM_OK;
}

aifmm_status aifmm_grid_points(aifmm_problem* p, double* xy) {
  if (!p || !xy) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    p->sync();
    p->d2h(xy, p->d_pts, sizeof(double2) * p->N);
  });
}

aifmm_status aifmm_rhs_plane_wave(aifmm_problem* p, int nrhs, const double* theta, double* b, int flags) {
  if (!p || !theta || !b || nrhs < 1) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    const double* dth = static_cast<const double*>(p->stage.put_raw(theta, sizeof(double) * nrhs, p->st));
    const size_t bytes = sizeof(double2) * (size_t)p->N * nrhs;
    const bool dev = flags & AIFMM_PTR_DEVICE;
    aifmm_problem::Tmp tb(p, dev ? 1 : bytes);
    double2* db = dev ? reinterpret_cast<double2*>(b) : tb.as<double2>();
    int e = aifmm_launch_rhs_plane_wave(p->d_pts, p->d_q, p->d.kappa, p->N, nrhs, dth, db, p->st);
    if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    if (!dev) CK(cudaMemcpyAsync(b, db, bytes, cudaMemcpyDeviceToHost, p->st));
    p->sync();
  });
}

aifmm_status aifmm_entries(aifmm_problem* p, long n, const int* I, const int* J, double* out, int flags) {
  if (!p || n < 0 || (n > 0 && (!I || !J || !out))) return AIFMM_ERR_ARG;
  if (!p->tables_ready) { p->err = "tables not ready"; return AIFMM_ERR_STATE; }
  return guard(p, [&] {
    if (n == 0) return;
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const int *dI = I, *dJ = J;
    double2* dO = reinterpret_cast<double2*>(out);
    if (!dev)
      for (long t = 0; t < n; ++t)
        if (I[t] < 0 || I[t] >= p->N || J[t] < 0 || J[t] >= p->N) throw Fail(AIFMM_ERR_ARG, "point index out of range");
    aifmm_problem::Tmp tI(p, dev ? 1 : sizeof(int) * n), tJ(p, dev ? 1 : sizeof(int) * n);
    aifmm_problem::Tmp tO(p, dev ? 1 : sizeof(double2) * n);
    if (!dev) {
      CK(cudaMemcpyAsync(tI.ptr, I, sizeof(int) * n, cudaMemcpyHostToDevice, p->st));
      CK(cudaMemcpyAsync(tJ.ptr, J, sizeof(int) * n, cudaMemcpyHostToDevice, p->st));
      dI = tI.as<int>(); dJ = tJ.as<int>(); dO = tO.as<double2>();
    }
    int e = aifmm_launch_list_entries(dI, dJ, n, dO, p->ctx(), p->st);
    if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    if (!dev) CK(cudaMemcpyAsync(out, dO, sizeof(double2) * n, cudaMemcpyDeviceToHost, p->st));
    p->sync();
  });
}

aifmm_status aifmm_get_matrix(aifmm_problem* p, int nr, const int* rows, int nc, const int* cols, double* out,
                              int flags) {
  if (!p || nr < 0 || nc < 0 || (nr * (long)nc > 0 && (!rows || !cols || !out))) return AIFMM_ERR_ARG;
  if (!p->tables_ready) { p->err = "tables not ready"; return AIFMM_ERR_STATE; }
  if (flags & AIFMM_PTR_DEVICE) {
    return guard(p, [&] {
      BlockDesc bd{rows, cols, nr, nc, reinterpret_cast<double2*>(out), nr, 0};
      std::vector<BlockDesc> v{bd};
      p->launch_blocks(v);
      p->sync();
    });
  }
  std::vector<int> I((size_t)nr * nc), J((size_t)nr * nc);
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r) { I[r + (size_t)c * nr] = rows[r]; J[r + (size_t)c * nr] = cols[c]; }
  return aifmm_entries(p, (long)nr * nc, I.data(), J.data(), out, AIFMM_PTR_HOST);
}

aifmm_status aifmm_build_tree(aifmm_problem* p) {
  if (!p) return AIFMM_ERR_ARG;
  return guard(p, [&] { p->build_tree(); });
}

aifmm_status aifmm_assemble(aifmm_problem* p) {
  if (!p) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    if (p->have_saved) { p->release_saved(); }
    p->have_saved = false;
    p->consumed = false;
    p->release_level_data();
    p->assemble();
  });
}

aifmm_status aifmm_factorize_solve(aifmm_problem* p, int nrhs, const double* b, double* x, int flags) {
  if (!p || !b || !x || nrhs < 1) return AIFMM_ERR_ARG;
  return guard(p, [&] { p->factorize_solve(nrhs, b, x, flags); });
}

aifmm_status aifmm_factorize(aifmm_problem* p, int precision, int flags) {
  if (!p) return AIFMM_ERR_ARG;
  if (precision != AIFMM_PRECISION_FP64 && precision != AIFMM_PRECISION_C64) {
    p->err = "precision must be AIFMM_PRECISION_FP64 or AIFMM_PRECISION_C64";
    return AIFMM_ERR_ARG;
  }
  return guard(p, [&] { p->factorize(flags, precision); });
}

aifmm_status aifmm_solve(aifmm_problem* p, int nrhs, const double* b, long ldb, double* x, long ldx, void* stream,
                         int flags) {
  if (!p || !b || !x || nrhs < 1) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if (cs) {  // the solve starts after the work already queued on the caller's stream
      CK(cudaEventRecord(p->ev_fork, cs));
      CK(cudaStreamWaitEvent(p->st, p->ev_fork, 0));
    }
    p->solve_rhs(nrhs, b, ldb, x, ldx, flags);
    p->st_back_ms = p->ms_solve;
    if (cs) {  // and the caller's stream sees the solution
      CK(cudaEventRecord(p->ev_join, p->st));
      CK(cudaStreamWaitEvent(cs, p->ev_join, 0));
    }
  });
}

aifmm_status aifmm_autotune(aifmm_problem* p, double* ms, int* tile_cols) {
  if (!p) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    p->autotune();
    if (ms) for (int i = 0; i < 4; ++i) ms[i] = p->tune_ms[i / 2][i % 2];
    if (tile_cols) { tile_cols[0] = p->gemm_cols[0]; tile_cols[1] = p->gemm_cols[1]; }
  });
}

aifmm_status aifmm_set_factor_tolerance(aifmm_problem* p, int tol_pow) {
  if (!p || tol_pow < 0 || tol_pow > 15) return AIFMM_ERR_ARG;
  p->tol_factor = tol_pow == 0 ? p->tol : std::pow(10, -1.0 * tol_pow);
  return AIFMM_OK;
}

aifmm_status aifmm_compressed_matvec(aifmm_problem* p, int nrhs, const double* x, long ldx, double* y, long ldy,
                                     int flags) {
  if (!p || !x || !y || nrhs < 1) return AIFMM_ERR_ARG;
  if (ldx < p->N || ldy < p->N) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const long N = p->N;
    const size_t bytes = sizeof(double2) * (size_t)N * nrhs;
    aifmm_problem::Tmp tx(p, dev ? 1 : bytes), ty(p, dev ? 1 : bytes);
    const double2* dx = reinterpret_cast<const double2*>(x);
    double2* dy = reinterpret_cast<double2*>(y);
    long lx = ldx, ly = ldy;
    if (!dev) {
      CK(cudaMemcpy2DAsync(tx.ptr, sizeof(double2) * N, x, sizeof(double2) * ldx, sizeof(double2) * N, nrhs,
                           cudaMemcpyHostToDevice, p->st));
      dx = tx.as<double2>(); dy = ty.as<double2>();
      lx = ly = N;
    }
    p->cur = p->st;
    p->nrhs = nrhs;
    p->compressed_matvec(dx, lx, dy, ly, nrhs);
    if (!dev)
      CK(cudaMemcpy2DAsync(y, sizeof(double2) * ldy, dy, sizeof(double2) * N, sizeof(double2) * N, nrhs,
                           cudaMemcpyDeviceToHost, p->st));
    p->sync();
  });
}

aifmm_status aifmm_solve_refined(aifmm_problem* p, int nrhs, const double* b, long ldb, double* x, long ldx,
                                 double rtol, int maxit, int* iterations, double* relres, int flags) {
  if (!p || !b || !x || nrhs < 1) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    p->cur = p->st;
    // the Krylov basis (31 vectors of N x nrhs) goes back to the device afterwards
    auto give_back = [&] {
      cudaStreamSynchronize(p->st);
      cudaStreamSynchronize(p->st2);
      p->pool.commit_frees();
      p->pool.release_free_big();
    };
    try {
      p->refine_solve(nrhs, b, ldb, x, ldx, flags, rtol, maxit, 30);
    } catch (...) {
      if (iterations) *iterations = p->gm_iters;
      if (relres) *relres = p->gm_relres;
      give_back();
      throw;
    }
    give_back();
    if (iterations) *iterations = p->gm_iters;
    if (relres) *relres = p->gm_relres;
  });
}

aifmm_status aifmm_find_error(aifmm_problem* p, int nrhs, const double* x, long ldx, const double* x_true, long ldt,
                              double* rel, int flags) {
  if (!p || !x || !x_true || !rel || nrhs < 1) return AIFMM_ERR_ARG;
  if (ldx < p->N || ldt < p->N) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    const long N = p->N;
    double se = 0.0, st = 0.0;
    if (flags & AIFMM_PTR_DEVICE) {
      aifmm_problem::Tmp part(p, aifmm_error_norms_scratch_bytes()), out(p, 2 * sizeof(double));
      int e = aifmm_launch_error_norms(reinterpret_cast<const double2*>(x), ldx,
                                       reinterpret_cast<const double2*>(x_true), ldt, N, nrhs, part.as<double>(),
                                       out.as<double>(), p->st);
      if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
      double h[2];
      CK(cudaMemcpyAsync(h, out.ptr, sizeof h, cudaMemcpyDeviceToHost, p->st));
      p->sync();
      se = h[0];
      st = h[1];
    } else {
      for (int c = 0; c < nrhs; ++c)
        for (long i = 0; i < N; ++i) {
          const double* a = x + 2 * (i + c * ldx);
          const double* t = x_true + 2 * (i + c * ldt);
          se += (a[0] - t[0]) * (a[0] - t[0]) + (a[1] - t[1]) * (a[1] - t[1]);
          st += t[0] * t[0] + t[1] * t[1];
        }
    }
    *rel = std::sqrt(se) / std::sqrt(st);
  });
}

aifmm_status aifmm_trim(aifmm_problem* p) {
  if (!p) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    p->sync();
    CK(cudaStreamSynchronize(p->st2));
    p->gb_idx.release(); p->gb_lst.release(); p->gb_segs.release();
    p->gb_ws.release(); p->gb_res.release(); p->gb_lu.release(); p->gb_acf.release();
    // the complex128 assembly of a complex64 factorisation is what its refined
    // solves multiply with: it stays
    if (p->have_saved && !(p->factored && p->factor_es == 8)) {
      p->release_saved();
      p->have_saved = false;
    }
    p->pool.commit_frees();
    p->pool.release_free_big();
  });
}

aifmm_status aifmm_zgemm(aifmm_problem* p, int opA, int opB, int m, int n, int k, const double* alpha,
                         const double* A, int lda, const double* B, int ldb, const double* beta, double* C, int ldc,
                         int flags) {
  if (!p || !alpha || !beta || m < 0 || n < 0 || k < 0 || (opA != 0 && opA != 1) || (opB != 0 && opB != 1))
    return AIFMM_ERR_ARG;
  const int ar = opA ? k : m, ac = opA ? m : k, br = opB ? n : k, bc = opB ? k : n;
  if (lda < std::max(1, ar) || ldb < std::max(1, br) || ldc < std::max(1, m)) return AIFMM_ERR_ARG;
  if ((long)m * n > 0 && (!C || ((long)k > 0 && (!A || !B)))) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    if ((long)m * n == 0) return;
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const size_t bA = sizeof(double2) * (size_t)lda * ac, bB = sizeof(double2) * (size_t)ldb * bc;
    const size_t bC = sizeof(double2) * (size_t)ldc * n;
    aifmm_problem::Tmp tA(p, dev ? 1 : bA), tB(p, dev ? 1 : bB), tC(p, dev ? 1 : bC);
    double2* dA = reinterpret_cast<double2*>(const_cast<double*>(A));
    double2* dB = reinterpret_cast<double2*>(const_cast<double*>(B));
    double2* dC = reinterpret_cast<double2*>(C);
    if (!dev) {
      if (k > 0) {
        CK(cudaMemcpyAsync(tA.ptr, A, bA, cudaMemcpyHostToDevice, p->st));
        CK(cudaMemcpyAsync(tB.ptr, B, bB, cudaMemcpyHostToDevice, p->st));
      }
      CK(cudaMemcpyAsync(tC.ptr, C, bC, cudaMemcpyHostToDevice, p->st));
      dA = tA.as<double2>(); dB = tB.as<double2>(); dC = tC.as<double2>();
    }
    Blk a{dA, ar, ac, lda}, b{dB, br, bc, ldb}, c{dC, m, n, ldc};
    p->cur = p->st;
    p->gemm(c, a, opA, b, opB, make_double2(alpha[0], alpha[1]), make_double2(beta[0], beta[1]));
    p->flush_gemm();
    if (!dev) CK(cudaMemcpyAsync(C, dC, bC, cudaMemcpyDeviceToHost, p->st));
    p->sync();
  });
}

aifmm_status aifmm_release_workspaces(aifmm_problem* p) {
  if (!p) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    p->sync();
    CK(cudaStreamSynchronize(p->st2));
    p->gb_idx.release(); p->gb_lst.release(); p->gb_segs.release();
    p->gb_ws.release(); p->gb_res.release(); p->gb_lu.release(); p->gb_acf.release();
    p->pool.commit_frees();
    p->pool.release_free_big();
  });
}

aifmm_status aifmm_dense_matvec(aifmm_problem* p, int nrhs, const double* x, double* y, int flags) {
  if (!p || !x || !y || nrhs < 1 || nrhs > 8) return AIFMM_ERR_ARG;
  if (!p->tables_ready) { p->err = "tables not ready"; return AIFMM_ERR_STATE; }
  return guard(p, [&] {
    const size_t bytes = sizeof(double2) * (size_t)p->N * nrhs;
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const double2* dx = reinterpret_cast<const double2*>(x);
    double2* dy = reinterpret_cast<double2*>(y);
    aifmm_problem::Tmp tx(p, dev ? 1 : bytes), ty(p, dev ? 1 : bytes);
    if (!dev) {
      CK(cudaMemcpyAsync(tx.ptr, x, bytes, cudaMemcpyHostToDevice, p->st));
      dx = tx.as<double2>(); dy = ty.as<double2>();
    }
    int e = aifmm_launch_dense_matvec(dx, dy, p->N, nrhs, p->ctx(), p->st);
    if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    if (!dev) CK(cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, p->st));
    p->sync();
  });
}

aifmm_status aifmm_total_field(aifmm_problem* p, int nrhs, const double* theta, const double* phi, double* u,
                               int flags) {
  if (!p || !theta || !phi || !u || nrhs < 1 || nrhs > 8) return AIFMM_ERR_ARG;
  if (!p->tables_ready) { p->err = "tables not ready"; return AIFMM_ERR_STATE; }
  return guard(p, [&] {
    const size_t bytes = sizeof(double2) * (size_t)p->N * nrhs;
    const bool dev = flags & AIFMM_PTR_DEVICE;
    const double2* dphi = reinterpret_cast<const double2*>(phi);
    double2* du = reinterpret_cast<double2*>(u);
    aifmm_problem::Tmp tphi(p, dev ? 1 : bytes), tu(p, dev ? 1 : bytes);
    if (!dev) {
      CK(cudaMemcpyAsync(tphi.ptr, phi, bytes, cudaMemcpyHostToDevice, p->st));
      dphi = tphi.as<double2>(); du = tu.as<double2>();
    }
    const double* dth = static_cast<const double*>(p->stage.put_raw(theta, sizeof(double) * nrhs, p->st));
    int e = aifmm_launch_incident_field(p->d_pts, p->d.kappa, p->N, nrhs, dth, du, p->st);
    if (!e) e = aifmm_launch_green_matvec_add(dphi, du, p->N, nrhs, p->ctx(), p->st);
    if (e) throw Fail(AIFMM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    if (!dev) CK(cudaMemcpyAsync(u, du, bytes, cudaMemcpyDeviceToHost, p->st));
    p->sync();
  });
}

aifmm_status aifmm_level_ranks(aifmm_problem* p, int level, int* rank_in, int* rank_out) {
  if (!p || !rank_in || !rank_out) return AIFMM_ERR_ARG;
  if (!p->assembled || level < 2 || level > p->depth) return AIFMM_ERR_STATE;
  for (int k = 0; k < p->nBoxes[level]; ++k) { rank_in[k] = p->T[level][k].rank_in; rank_out[k] = p->T[level][k].rank_out; }
  return AIFMM_OK;
}

aifmm_status aifmm_box_skeleton(aifmm_problem* p, int level, int box, int which, int* out, int cap, int* count) {
  if (!p || !count || (cap > 0 && !out)) return AIFMM_ERR_ARG;
  if (!p->assembled || level < 2 || level > p->depth || box < 0 || box >= p->nBoxes[level]) return AIFMM_ERR_STATE;
  const Box& b = p->T[level][box];
  const std::vector<int>* v = which == 0 ? &b.in_check : which == 1 ? &b.in_charge : which == 2 ? &b.out_check : &b.out_charge;
  *count = (int)v->size();
  for (int i = 0; i < *count && i < cap; ++i) out[i] = (*v)[i];
  return AIFMM_OK;
}

aifmm_status aifmm_phase_times(const aifmm_problem* p, double* ms) {
  if (!p || !ms) return AIFMM_ERR_ARG;
  for (int i = 0; i < 4; ++i) ms[i] = p->ms[i];
  ms[4] = p->ms_factor;
  ms[5] = p->ms_solve;
  return AIFMM_OK;
}

aifmm_status aifmm_launch_counts(const aifmm_problem* p, long* factor_solve, long* assemble) {
  if (!p || !factor_solve || !assemble) return AIFMM_ERR_ARG;
  *factor_solve = p->launches_fs;
  *assemble = p->launches_asm;
  return AIFMM_OK;
}

aifmm_status aifmm_launch_counts_split(const aifmm_problem* p, long* factorize, long* solve) {
  if (!p || !factorize || !solve) return AIFMM_ERR_ARG;
  *factorize = p->launches_factor;
  *solve = p->launches_solve;
  return AIFMM_OK;
}

aifmm_status aifmm_kernel_profile(aifmm_problem* p, int kind, int enable) {
  if (!p || kind < 0 || kind >= aifmm_problem::kKinds) return AIFMM_ERR_ARG;
  p->prof_on[kind] = enable != 0;
  p->prof_launches[kind] = 0;
  p->prof_ms[kind] = 0;
  p->prof_flops[kind] = 0;
  return AIFMM_OK;
}

aifmm_status aifmm_kernel_profile_read(aifmm_problem* p, int kind, long* launches, double* ms, double* flops) {
  if (!p || !launches || !ms || !flops || kind < 0 || kind >= aifmm_problem::kKinds) return AIFMM_ERR_ARG;
  return guard(p, [&] {
    p->prof_collect();
    *launches = p->prof_launches[kind];
    *ms = p->prof_ms[kind];
    *flops = p->prof_flops[kind];
  });
}

aifmm_status aifmm_stats(const aifmm_problem* p, double* out, int n) {
  if (!p || !out) return AIFMM_ERR_ARG;
  const double grow = (double)(p->gb_idx.capacity() + p->gb_lst.capacity() + p->gb_segs.capacity() +
                               p->gb_ws.capacity() + p->gb_res.capacity() + p->gb_lu.capacity() +
                               p->gb_acf.capacity() +
                               p->scratch.capacity() + p->stage.cap_);
  const double v[15] = {p->st_sync_ms, (double)p->st_syncs, p->st_pending_ms, p->st_elim_ms, p->st_back_ms,
                        (double)p->st_compress, p->ms[3], (double)p->launches_fs,
                        p->st_asm_lists_ms, p->st_asm_aca_ms, p->st_asm_lu_ms, p->st_asm_blocks_ms,
                        p->st_asm_aca_gpu_ms, (double)p->pool.reserved(), grow};
  for (int i = 0; i < n && i < 15; ++i) out[i] = v[i];
  return AIFMM_OK;
}

aifmm_status aifmm_get_stream(const aifmm_problem* p, void** stream) {
  if (!p || !stream) return AIFMM_ERR_ARG;
  *stream = (void*)p->st;
  return AIFMM_OK;
}

}  // extern "C"
