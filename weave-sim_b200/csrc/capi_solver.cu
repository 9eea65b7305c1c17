// C entry points of the solver: a context owns a batch of instances packed into one device arena, the host goals of
// every instance (for warm starts and downloads), a CUDA stream and the graph of the plain form.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/weavesim.h"
#include "dr_kernels.hpp"
#include "errors.hpp"
#include "host_goals.hpp"
#include "tune.hpp"

using namespace wsb;

namespace {

struct CudaError : std::runtime_error { using std::runtime_error::runtime_error; };
#define CK(x)                                                                                                \
  do {                                                                                                       \
    cudaError_t e_ = (x);                                                                                    \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));                 \
  } while (0)

// element counts of the whole batch
struct Sizes { int n = 0, m = 0, p = 0, c = 0, k = 0, s = 0, b = 0; };   // b: instances (as an offset: the index)

// carves typed arrays out of one allocation (base == nullptr: only counts the bytes)
struct Carver {
  char *base;
  size_t off = 0;
  template <class T> T *take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
    off += sizeof(T) * std::max<size_t>(count, 1);
    return p;
  }
};

template <int P>
void layout(Dev<P> &d, Carver &cv, const Sizes &z) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A; using U = typename Dev<P>::U; using S = typename Dev<P>::S;
  d.ntot = z.n; d.mtot = z.m; d.ptot = z.p; d.ctot = z.c; d.ktot = z.k; d.stot = z.s;
  d.nS = z.n; d.xB = 3 * z.n; d.mS = z.m; d.qB = 4 * z.m; d.pS = z.p; d.cS = z.c; d.kS = z.k;
  d.sS = d.kB = d.oB = 2 * z.k; d.rB = z.m;
  const size_t n = z.n, m = z.m, p = z.p, c = z.c, k = z.k, s = z.s;
  d.X = cv.take<S>(6 * n); d.Xlo = PrecT<P>::TWO ? cv.take<S>(6 * n) : nullptr;
  d.V = cv.take<R>(3 * n); d.mass = cv.take<R>(n); d.lc = cv.take<R>(3 * n); d.ll = cv.take<R>(3 * n);
  d.nflag = cv.take<uint8_t>(n); d.nsOut = cv.take<int>(n); d.nsIn = cv.take<int>(n); d.anc = cv.take<int>(n);
  d.ancStart = cv.take<W>(3 * n); d.ancDelta = cv.take<W>(3 * n); d.react = cv.take<R>(3 * n);
  d.Q = cv.take<S>(8 * m); d.Qlo = PrecT<P>::TWO ? cv.take<S>(8 * m) : nullptr;
  d.Wr = cv.take<R>(3 * m);
  d.segI0 = cv.take<int>(m); d.segI1 = cv.take<int>(m); d.jA = cv.take<int>(m); d.jB = cv.take<int>(m);
  d.cl0 = cv.take<int>(m); d.cl1 = cv.take<int>(m); d.segStrand = cv.take<int>(m); d.segLocal = cv.take<int>(m);
  d.l0 = cv.take<R>(m); d.il0 = cv.take<W>(m); d.EA = cv.take<R>(m); d.GA = cv.take<R>(m); d.krs = cv.take<R>(3 * m);
  d.nF = cv.take<R>(3 * m); d.en = cv.take<R>(3 * m); d.Nax = cv.take<R>(m); d.Vsh = cv.take<R>(2 * m);
  d.rngLo = cv.take<int>(2 * m); d.rngHi = cv.take<int>(2 * m);
  d.jS0 = cv.take<int>(p); d.jS1 = cv.take<int>(p); d.jLen = cv.take<R>(p); d.EIx = cv.take<R>(p); d.EIy = cv.take<R>(p);
  d.GJ = cv.take<R>(p); d.om = cv.take<R>(3 * p); d.tau = cv.take<R>(3 * p); d.kd = cv.take<R>(3 * p); d.Mj = cv.take<R>(3 * p);
  d.cSeg = cv.take<int>(c); d.cLen = cv.take<R>(c); d.cB = cv.take<R>(3 * c); d.cQ = cv.take<W>(4 * c);
  d.tauC = cv.take<R>(3 * c); d.cM = cv.take<R>(2 * c);
  d.cxSegOff = cv.take<int>(2 * k); d.cxNseg = cv.take<int>(2 * k); d.cxNodeOff = cv.take<int>(2 * k); d.wk = cv.take<R>(2 * k); d.hk = cv.take<R>(2 * k);
  d.cw = cv.take<R>(k); d.ch = cv.take<R>(k); d.mu = cv.take<R>(k); d.cflag = cv.take<uint8_t>(k);
  d.u = cv.take<U>(2 * k); d.nPrev = cv.take<R>(3 * k); d.slip = cv.take<A>(k); d.stuck = cv.take<uint8_t>(k);
  d.cstate = cv.take<uint8_t>(k); d.Fn = cv.take<R>(k); d.Ft = cv.take<R>(k); d.gap = cv.take<R>(k);
  d.sPos = cv.take<int>(2 * k); d.sKey = cv.take<int>(4 * k); d.sInv = cv.take<int>(4 * k); d.sKeyS = cv.take<int>(2 * k);
  d.sSideAt = cv.take<int>(2 * k);
  d.sStrand = cv.take<int>(2 * k); d.sT = cv.take<R>(2 * k);
  d.kth = cv.take<R>(2 * k); d.sF = cv.take<R>(6 * k); d.sTq = cv.take<R>(6 * k);
  d.stSideOff = cv.take<int>(s); d.stSideCnt = cv.take<int>(s); d.stSegOff = cv.take<int>(s);
  d.ord = cv.take<int>(4 * k); d.ordSeg = cv.take<int>(4 * k);
  d.fc90 = cv.take<R>(2 * k); d.E90 = cv.take<R>(2 * k); d.Hs = cv.take<R>(2 * k); d.sProj = cv.take<R>(4 * k); d.sinT = cv.take<R>(k);
  d.ctype = cv.take<uint8_t>(k); d.theta = cv.take<R>(k); d.area = cv.take<R>(k); d.pres = cv.take<R>(k);
  d.util = cv.take<R>(k); d.phiS = cv.take<R>(2 * k);
  d.flW = cv.take<R>(n); d.flH = cv.take<R>(n); d.flAx = cv.take<W>(n); d.flAy = cv.take<W>(n);
  d.flF = cv.take<R>(3 * n); d.flState = cv.take<uint8_t>(n); d.ldTot = cv.take<R>(3 * n);
  d.nodeJoint = cv.take<int>(n); d.nodeClamp = cv.take<int>(n); d.X0 = cv.take<W>(3 * n);
  d.segM = cv.take<R>(3 * m); d.nodeLay = cv.take<R>(4 * n);
  d.utmSched = cv.take<double>(WS_PROTOCOL_MAX_INC * size_t(std::max(z.b, 1)));
  d.utmOut = cv.take<double>(4 * WS_PROTOCOL_MAX_INC * size_t(std::max(z.b, 1)));
  d.ext = cv.take<InstExt>(size_t(std::max(z.b, 1)));
  d.lam = cv.take<A>(k); d.penAcc = cv.take<A>(k); d.dent = cv.take<R>(2 * k); d.climb = cv.take<R>(2 * k);
  d.tanpsi = cv.take<R>(2 * k); d.dentE = cv.take<R>(k); d.theta0 = cv.take<R>(k); d.Mrot = cv.take<R>(k);
  d.rotSlip = cv.take<A>(k);
}

// host -> device with conversion, batched: put() converts into a host buffer and queues the copy; flushPuts() sends the
// queue through the context's staging buffer with one synchronisation.  Every entry point that puts flushes before it
// returns (and a failed one drops its queue), so nothing queued outlives the call that queued it.
struct PendingPut { void *dst; size_t off, bytes; };
thread_local std::vector<char> t_putHost;
thread_local std::vector<PendingPut> t_puts;
template <class T, class V>
void put(T *dst, const V *src, size_t count, cudaStream_t) {
  if (!count) return;
  const size_t off = t_putHost.size(), bytes = count * sizeof(T);
  t_putHost.resize(off + ((bytes + 15) & ~size_t(15)));
  T *h = reinterpret_cast<T *>(t_putHost.data() + off);
  for (size_t i = 0; i < count; i++) h[i] = T(src[i]);
  t_puts.push_back({dst, off, bytes});
}
void dropPuts() { t_puts.clear(); t_putHost.clear(); }
template <class T>
void getv(std::vector<double> &out, const T *src, size_t count, cudaStream_t st) {
  std::vector<T> tmp(count);
  if (count) CK(cudaMemcpyAsync(tmp.data(), src, count * sizeof(T), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  out.resize(count);
  for (size_t i = 0; i < count; i++) out[i] = double(tmp[i]);
}

}  // namespace

struct ws_ctx {
  int prec = 0, form = 0, threads = 0, device = 0;
  cudaStream_t st = nullptr;
  std::vector<HostGoals> g;
  std::vector<InstDesc> inst;
  std::vector<int> order;
  Sizes z;
  char *arena = nullptr;
  size_t bytes = 0;
  Dev<PREC_F64> d64{};
  Dev<PREC_MIXED> dmx{};
  Dev<PREC_F32> d32{};
  InstDesc *dInst = nullptr;
  InstCtl *dCtl = nullptr;
  InstExt *dExt = nullptr;         // the load protocols' state (in the arena)
  std::vector<InstExt> extHost;
  int *dOrder = nullptr;         // batched form: the instances of the one-block kernels, longest first
  int nNarrow = 0;               // ... and their count
  std::vector<char> isWide;      // per instance
  std::vector<uint8_t> ranLast;  // per instance: selected by the last ws_step's mask
  int *dWide = nullptr;          // batched form: the wide instances (a cluster each), longest first
  int nWide = 0;
  int wideCl = 0;                // blocks in a wide instance's cluster (0: no wide instances)
  int wideMin = 0;               // nodes + segments from which an instance is wide
  cudaStream_t sideCta = nullptr;            // batched form: the one-block kernels beside the cluster kernel
  cudaEvent_t ctaFork = nullptr, ctaJoin = nullptr;
  uint8_t *dMask = nullptr;
  void *dPart = nullptr;
  unsigned *dBar = nullptr;   // grid form: barrier counter + generation, and its timeout flag
  int *dErr = nullptr;
  int gridBlocks[2][2] = {{0, 0}, {0, 0}};   // grid form: co-resident blocks [short-slide side order][extensions]
  PlainShape shape{};
  int sidesGeneral = 0;          // ws_opts.side_order == WS_SIDES_GENERAL
  int ctaGlobal = 0;             // ws_opts.cta_state == WS_CTA_GLOBAL
  size_t residentBytes = 0;      // batched form: dynamic shared memory of the resident form (0: global state)
  bool shortSides = false;       // the short-slide side order is in use
  cudaGraphExec_t graph = nullptr;
  int graphIters = 0, graphKey = -1, graphLaunches = 0;
  PlainFork fork{};              // plain form: the crossing kernel's stream and the fork / join events
  int plainMode = 0;             // plain form: 0 forked graph branches, 1 one launch a phase with block roles, 2 one kernel a phase
  ws_shape launch{};             // the launch shape in use (ws_get_shape)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evChunk[8] = {};   // pipelined downloads: one per chunk of the device-to-host copy
  double lastMs = 0;
  int64_t lastLaunches = 0;
  std::vector<InstCtl> ctlHost;
  // host staging of uploads / downloads: pinned (cudaMallocHost) in contexts made by ws_create, an ordinary host vector
  // in the allocation-free entry point's temporary context
  bool pinnedOK = false;
  char *pinned = nullptr;
  size_t pinnedCap = 0;
  std::vector<char> pageable;
  unsigned char *dXfer = nullptr;   // device side of uploads / downloads (contexts made by ws_create)
  size_t xferCap = 0;
};

namespace {

// A transfer through the pinned staging buffer in chunks, so that the host's copy of one chunk overlaps the DMA of
// another (one core's memcpy, about 15 GB/s, takes longer than the PCIe copy).  A piece is a caller's array and its
// byte offset in the staging buffer.
struct Piece { char *user; size_t off, bytes; };
constexpr int kChunks = 8;
constexpr size_t kChunkMin = 512 * 1024;

int chunkCount(size_t bytes) { return int(std::max<size_t>(1, std::min<size_t>(kChunks, bytes / kChunkMin))); }
size_t chunkEdge(size_t bytes, int nc, int k) {
  const size_t step = ((bytes + nc - 1) / nc + 15) & ~size_t(15);
  return std::min(bytes, step * size_t(k));
}
// copies the parts of the pieces inside staging bytes [lo, hi): into the staging buffer (toStage) or out of it
void copyRange(const std::vector<Piece> &ps, char *stage, size_t lo, size_t hi, bool toStage) {
  for (const Piece &q : ps) {
    const size_t a = std::max(lo, q.off), e = std::min(hi, q.off + q.bytes);
    if (a >= e) continue;
    if (toStage) std::memcpy(stage + a, q.user + (a - q.off), e - a);
    else std::memcpy(q.user + (a - q.off), stage + a, e - a);
  }
}

char *stageBuf(ws_ctx *c, size_t bytes) {
  if (!c->pinnedOK) {
    if (c->pageable.size() < bytes) c->pageable.resize(bytes);
    return c->pageable.data();
  }
  if (c->pinnedCap < bytes) {
    if (c->pinned) CK(cudaFreeHost(c->pinned));
    c->pinned = nullptr;
    c->pinnedCap = 0;
    CK(cudaMallocHost(&c->pinned, bytes));
    c->pinnedCap = bytes;
  }
  return c->pinned;
}

unsigned char *xferBuf(ws_ctx *c, size_t bytes) {
  if (c->xferCap < bytes) {
    if (c->dXfer) CK(cudaFree(c->dXfer));
    c->dXfer = nullptr;
    c->xferCap = 0;
    CK(cudaMalloc(&c->dXfer, bytes));
    c->xferCap = bytes;
  }
  return c->dXfer;
}

void flushPuts(ws_ctx *c) {
  if (t_puts.empty()) return;
  char *buf = stageBuf(c, t_putHost.size());
  std::memcpy(buf, t_putHost.data(), t_putHost.size());
  for (const PendingPut &q : t_puts) CK(cudaMemcpyAsync(q.dst, buf + q.off, q.bytes, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  dropPuts();
}

// device -> host in one go: planes are queued, copied asynchronously into the staging buffer, and converted to the
// caller's interleaved f64 (or byte) arrays after a single synchronisation
struct Fetch {
  struct Item { const void *src; size_t bytes, off; std::function<void(const char *)> put; };
  std::vector<Item> items;
  size_t total = 0;
  std::deque<std::vector<double>> tmp;         // host scratch of fields derived from several planes
  std::vector<std::function<void()>> after;    // run once the planes have landed
  double *scratch(size_t n) { tmp.emplace_back(n); return tmp.back().data(); }
  template <class T>
  void planes(const T *base, size_t stride, size_t first, size_t count, int ncomp, double *dst) {
    for (int k = 0; k < ncomp; k++) {
      const size_t off = total;
      total += (count * sizeof(T) + 15) & ~size_t(15);
      items.push_back({base + size_t(k) * stride + first, count * sizeof(T), off, [=](const char *p) {
                         const T *v = reinterpret_cast<const T *>(p);
                         for (size_t i = 0; i < count; i++) dst[size_t(ncomp) * i + k] = double(v[i]);
                       }});
    }
  }
  // two-float planes: hi and lo added in f64
  template <class T>
  void pairs(const T *hi, const T *lo, size_t stride, size_t first, size_t count, int ncomp, double *dst) {
    for (int k = 0; k < ncomp; k++) {
      const size_t oh = total;
      total += (count * sizeof(T) + 15) & ~size_t(15);
      const size_t ol = total;
      if (lo) total += (count * sizeof(T) + 15) & ~size_t(15);
      items.push_back({hi + size_t(k) * stride + first, count * sizeof(T), oh, nullptr});
      if (lo) items.push_back({lo + size_t(k) * stride + first, count * sizeof(T), ol, nullptr});
      const bool two = lo != nullptr;
      items.back().put = [=](const char *p0) {
        const T *h = reinterpret_cast<const T *>(p0 - (two ? ol : oh) + oh);
        const T *l = two ? reinterpret_cast<const T *>(p0) : nullptr;
        for (size_t i = 0; i < count; i++) dst[size_t(ncomp) * i + k] = double(h[i]) + (two ? double(l[i]) : 0.0);
      };
    }
  }
  void bytes(const uint8_t *src, size_t count, uint8_t *dst) {
    const size_t off = total;
    total += (count + 15) & ~size_t(15);
    items.push_back({src, count, off, [=](const char *p) { std::memcpy(dst, p, count); }});
  }
  void run(ws_ctx *c) {
    char *buf = stageBuf(c, std::max<size_t>(total, 16));
    for (auto &it : items) if (it.bytes) CK(cudaMemcpyAsync(buf + it.off, it.src, it.bytes, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (auto &it : items) if (it.put) it.put(buf + it.off);
    for (auto &f : after) f();
  }
};

template <int P> Dev<P> &devOf(ws_ctx *c);
template <> Dev<PREC_F64> &devOf<PREC_F64>(ws_ctx *c) { return c->d64; }
template <> Dev<PREC_MIXED> &devOf<PREC_MIXED>(ws_ctx *c) { return c->dmx; }
template <> Dev<PREC_F32> &devOf<PREC_F32>(ws_ctx *c) { return c->d32; }

InstDesc describe(const HostGoals &g, const Sizes &off) {
  InstDesc I{};
  I.n0 = off.n; I.n = g.n; I.m0 = off.m; I.m = g.m; I.p0 = off.p; I.p = g.p; I.c0 = off.c; I.C = g.C;
  I.k0 = off.k; I.K = g.K; I.s0 = off.s; I.S = g.S;
  I.warmup = g.prm.warmup_iter; I.ramp_iter = std::max(g.prm.ramp_iter, 0); I.disp_ramp = std::max(g.prm.disp_ramp_iter, 0);
  I.kd = g.prm.kinetic_damping ? 1 : 0; I.contacts = g.prm.contacts ? 1 : 0; I.max_iter = g.prm.max_iter > 0 ? g.prm.max_iter : 0x7fffffff;
  I.localLoads = 0;
  for (uint8_t h : g.hasLocal) I.localLoads |= h ? 1 : 0;
  I.ms = g.prm.mass_scale; I.damping = g.prm.damping; I.tol = g.prm.tol; I.strength = g.prm.strength; I.stick = g.prm.stick_strength;
  I.tf = g.prm.torsion_factor; I.eps = g.prm.epsilon; I.slip_rate = g.prm.slip_rate; I.lRef = g.lRef; I.jLenMin = g.jLenMin;
  I.edgeThr = g.prm.edge_threshold;
  I.aug = g.prm.augmented ? 1 : 0; I.alEvery = g.prm.al_every; I.rotFric = g.prm.rot_friction ? 1 : 0;
  I.seat = g.prm.seat_law ? 1 : 0; I.seatGap = g.prm.seat_gap ? 1 : 0;
  I.dentAfter = g.prm.dent_after_iter >= 0 ? g.prm.dent_after_iter : g.dentAfterDefault;
  I.rotFactor = g.prm.rot_factor; I.dentRate = g.prm.dent_rate;
  I.ext = (I.aug || I.rotFric || I.seat) ? 1 : 0;
  I.utmMode = g.proto.mode; I.utmProbe = off.n + g.proto.probe; I.utmNInc = g.proto.n_inc; I.utmSettle = g.proto.settle;
  I.utmAvg = g.proto.avg; I.utmIdx = off.b;
  I.cxLin = g.cxLinear ? 1 : 0;
  I.floorOn = g.prm.floor ? 1 : 0; I.floorZ = g.prm.floor_z; I.floorMu = g.prm.floor_mu;
  I.rbOn = g.rigid ? 1 : 0; I.rbR = g.rbR; I.rbVmax = g.rbVmax; I.rbWmax = g.rbWmax;
  for (int k = 0; k < 3; k++) I.utmAxis[k] = g.proto.axis[k];
  return I;
}

// the load protocol's state at its start: settling, no increment recorded, the first value applied
InstExt protocolState(const HostGoals &g) {
  InstExt u{};
  u.curF = g.proto.mode ? g.proto.sched[0] : 0.0;
  for (int k = 0; k < 3; k++) {
    u.pf[k] = g.proto.mode == 1 ? g.proto.axis[k] * g.proto.sched[0] : 0.0;
    u.p0[k] = g.probe0[k];
  }
  return u;
}

// upload the goal arrays of instance b (everything a warm start may change)
template <int P>
void uploadGoals(ws_ctx *c, int b) {
  Dev<P> &d = devOf<P>(c);
  using R = typename Dev<P>::R; using W = typename Dev<P>::W;
  const HostGoals &g = c->g[b];
  const InstDesc &I = c->inst[b];
  cudaStream_t st = c->st;
  const size_t n = g.n, m = g.m, p = g.p, C = g.C, K = g.K;
  put<R>(d.mass + I.n0, g.mass.data(), n, st);
  for (int k = 0; k < 3; k++) {
    std::vector<double> a(n), l(n);
    for (size_t i = 0; i < n; i++) { a[i] = g.loadConst[3 * i + k]; l[i] = g.loadLocal[3 * i + k]; }
    put<R>(d.lc + size_t(k) * d.ntot + I.n0, a.data(), n, st);
    put<R>(d.ll + size_t(k) * d.ntot + I.n0, l.data(), n, st);
  }
  std::vector<uint8_t> fl(n);
  for (size_t i = 0; i < n; i++)
    fl[i] = (g.nodeFree[3 * i] ? 1 : 0) | (g.nodeFree[3 * i + 1] ? 2 : 0) | (g.nodeFree[3 * i + 2] ? 4 : 0) | (g.fixedAny[i] ? 8 : 0) |
            (g.hasLocal[i] ? 16 : 0) | (g.ancIndex[i] >= 0 ? 32 : 0);
  put<uint8_t>(d.nflag + I.n0, fl.data(), n, st);
  // prescribed motion: slot s of this instance lives at the instance's node offset + s
  std::vector<int> anc(n);
  for (size_t i = 0; i < n; i++) anc[i] = g.ancIndex[i] >= 0 ? I.n0 + g.ancIndex[i] : -1;
  put<int>(d.anc + I.n0, anc.data(), n, st);
  const size_t ns = g.ancStart.size() / 3;
  for (int k = 0; k < 3; k++) {
    std::vector<double> a(ns), dl(ns);
    for (size_t s = 0; s < ns; s++) { a[s] = g.ancStart[3 * s + k]; dl[s] = g.ancDelta[3 * s + k]; }
    put<W>(d.ancStart + size_t(k) * d.ntot + I.n0, a.data(), ns, st);
    put<W>(d.ancDelta + size_t(k) * d.ntot + I.n0, dl.data(), ns, st);
  }
  put<R>(d.EA + I.m0, g.EA.data(), m, st);
  put<R>(d.GA + I.m0, g.GA.data(), m, st);
  for (int k = 0; k < 3; k++) {
    std::vector<double> a(m);
    for (size_t j = 0; j < m; j++) a[j] = g.kRotStatic[3 * j + k];
    put<R>(d.krs + size_t(k) * d.mtot + I.m0, a.data(), m, st);
  }
  put<R>(d.EIx + I.p0, g.EIx.data(), p, st);
  put<R>(d.EIy + I.p0, g.EIy.data(), p, st);
  put<R>(d.GJ + I.p0, g.GJ.data(), p, st);
  for (int k = 0; k < 3; k++) {
    std::vector<double> a(p);
    for (size_t j = 0; j < p; j++) a[j] = g.omega0[3 * j + k];
    put<R>(d.om + size_t(k) * d.ptot + I.p0, a.data(), p, st);
  }
  std::vector<int> cs(C);
  for (size_t q = 0; q < C; q++) cs[q] = I.m0 + g.cSeg[q];
  put<int>(d.cSeg + I.c0, cs.data(), C, st);
  put<R>(d.cLen + I.c0, g.cLen.data(), C, st);
  for (int k = 0; k < 3; k++) {
    std::vector<double> a(C);
    for (size_t q = 0; q < C; q++) a[q] = g.cB[3 * q + k];
    put<R>(d.cB + size_t(k) * d.ctot + I.c0, a.data(), C, st);
  }
  for (int k = 0; k < 4; k++) {
    std::vector<double> a(C);
    for (size_t q = 0; q < C; q++) a[q] = g.cQ[4 * q + k];
    put<W>(d.cQ + size_t(k) * d.ctot + I.c0, a.data(), C, st);
  }
  std::vector<int> c0(m), c1(m);
  for (size_t j = 0; j < m; j++) { c0[j] = g.segClamp0[j] >= 0 ? I.c0 + g.segClamp0[j] : -1; c1[j] = g.segClamp1[j] >= 0 ? I.c0 + g.segClamp1[j] : -1; }
  put<int>(d.cl0 + I.m0, c0.data(), m, st);
  put<int>(d.cl1 + I.m0, c1.data(), m, st);
  put<R>(d.mu + I.k0, g.mu.data(), K, st);
  std::vector<uint8_t> cf(K);
  for (size_t q = 0; q < K; q++) cf[q] = (g.enabled[q] ? 1 : 0) | (g.locked[q] ? 2 : 0);
  put<uint8_t>(d.cflag + I.k0, cf.data(), K, st);
}

// upload the sorted side lists, segment slices and side keys (the segments the sides sit on now) of instance b into
// sorted-side buffer `buf`
template <int P>
void uploadOrder(ws_ctx *c, int b, int buf) {
  Dev<P> &d = devOf<P>(c);
  const HostGoals &g = c->g[b];
  const InstDesc &I = c->inst[b];
  const size_t K2 = 2 * size_t(d.ktot), K = g.K, m = g.m;
  std::vector<int> ord(2 * K), lo(m), hi(m), key(2 * K), inv(2 * K);
  for (size_t q = 0; q < 2 * K; q++) ord[q] = 2 * I.k0 + g.sidePos[g.ord[q]];
  for (size_t q = 0; q < 2 * K; q++) inv[g.sidePos[g.ord[q]]] = 2 * I.k0 + int(q);
  for (size_t q = 0; q < 2 * K; q++) key[q] = g.sideSegLocal(g.sideList[q]);
  for (size_t j = 0; j < m; j++) { lo[j] = 2 * I.k0 + g.rngLo[j]; hi[j] = 2 * I.k0 + g.rngHi[j]; }
  put<int>(d.sKey + buf * K2 + 2 * size_t(I.k0), key.data(), 2 * K, c->st);
  put<int>(d.ord + buf * K2 + 2 * size_t(I.k0), ord.data(), 2 * K, c->st);
  put<int>(d.sInv + buf * K2 + 2 * size_t(I.k0), inv.data(), 2 * K, c->st);
  put<int>(d.ordSeg + buf * K2 + 2 * size_t(I.k0), g.ordSeg.data(), 2 * K, c->st);
  put<int>(d.rngLo + size_t(buf) * d.mtot + I.m0, lo.data(), m, c->st);
  put<int>(d.rngHi + size_t(buf) * d.mtot + I.m0, hi.data(), m, c->st);
}

// positions / frames of instance b into buffer `buf` (and its slide coordinates): converted into the staging buffer,
// copied asynchronously, one synchronisation; velocities are cleared on the device
template <int P>
void uploadState(ws_ctx *c, int b, int buf, bool withU) {
  Dev<P> &d = devOf<P>(c);
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using S = typename Dev<P>::S; using U = typename Dev<P>::U;
  const HostGoals &g = c->g[b];
  const InstDesc &I = c->inst[b];
  cudaStream_t st = c->st;
  const size_t n = g.n, m = g.m, K = g.K;
  const int nS = PrecT<P>::TWO ? 2 : 1;
  auto al = [](size_t x) { return (x + 15) & ~size_t(15); };
  const size_t bytes = nS * (3 * al(n * sizeof(S)) + 4 * al(m * sizeof(S))) + (withU && K ? 2 * al(K * sizeof(U)) + 3 * al(K * sizeof(R)) : 0);
  char *sb = stageBuf(c, std::max<size_t>(bytes, 16));
  size_t off = 0;
  auto stagePlane = [&](auto *dst, size_t count, auto fill) {
    using T = std::remove_pointer_t<decltype(dst)>;
    T *h = reinterpret_cast<T *>(sb + off);
    for (size_t i = 0; i < count; i++) h[i] = fill(i);
    CK(cudaMemcpyAsync(dst, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    off += al(count * sizeof(T));
  };
  for (int k = 0; k < 3; k++) {
    stagePlane(d.X + size_t(buf * 3 + k) * d.ntot + I.n0, n, [&](size_t i) { return S(W(g.X[3 * i + k])); });
    if (PrecT<P>::TWO)
      stagePlane(d.Xlo + size_t(buf * 3 + k) * d.ntot + I.n0, n, [&](size_t i) { const W a = W(g.X[3 * i + k]); return S(a - W(S(a))); });
    CK(cudaMemsetAsync(d.V + size_t(k) * d.ntot + I.n0, 0, n * sizeof(R), st));
  }
  for (int k = 0; k < 4; k++) {
    stagePlane(d.Q + size_t(buf * 4 + k) * d.mtot + I.m0, m, [&](size_t j) { return S(W(g.Q[4 * j + k])); });
    if (PrecT<P>::TWO)
      stagePlane(d.Qlo + size_t(buf * 4 + k) * d.mtot + I.m0, m, [&](size_t j) { const W a = W(g.Q[4 * j + k]); return S(a - W(S(a))); });
  }
  for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(d.Wr + size_t(k) * d.mtot + I.m0, 0, m * sizeof(R), st));
  if (withU && K) {
    for (int side = 0; side < 2; side++) stagePlane(d.u + size_t(side) * d.ktot + I.k0, K, [&](size_t q) { return U(g.u[2 * q + side]); });
    for (int k = 0; k < 3; k++) stagePlane(d.nPrev + size_t(k) * d.ktot + I.k0, K, [&](size_t q) { return R(g.nPrev[3 * q + k]); });
  }
  CK(cudaStreamSynchronize(st));
}

// the displacement origin of instance b as the host goals hold it
template <int P>
void displacementOrigin(ws_ctx *c, int b) {
  Dev<P> &d = devOf<P>(c);
  using W = typename Dev<P>::W;
  const HostGoals &g = c->g[b];
  for (int k = 0; k < 3; k++) {
    std::vector<double> x0(g.n);
    for (int i = 0; i < g.n; i++) x0[i] = g.X0[3 * size_t(i) + k];
    put<W>(d.X0 + size_t(k) * d.ntot + c->inst[b].n0, x0.data(), g.n, c->st);
  }
}

// the section at every node of instance b, for the ground's clearance
template <int P>
void floorSections(ws_ctx *c, int b) {
  Dev<P> &d = devOf<P>(c);
  using R = typename Dev<P>::R;
  const HostGoals &g = c->g[b];
  if (g.nodeW.empty()) return;
  put<R>(d.flW + c->inst[b].n0, g.nodeW.data(), g.n, c->st);
  put<R>(d.flH + c->inst[b].n0, g.nodeH.data(), g.n, c->st);
}

// the static arrays of instance b (topology, rest state, section constants)
template <int P>
void uploadStatic(ws_ctx *c, int b) {
  Dev<P> &d = devOf<P>(c);
  using R = typename Dev<P>::R; using W = typename Dev<P>::W;
  const HostGoals &g = c->g[b];
  const InstDesc &I = c->inst[b];
  cudaStream_t st = c->st;
  const size_t n = g.n, m = g.m, p = g.p, K = g.K, S = g.S;
  auto shift = [](const std::vector<int> &v, int off) { std::vector<int> o(v.size()); for (size_t i = 0; i < v.size(); i++) o[i] = v[i] >= 0 ? v[i] + off : -1; return o; };
  put<int>(d.nsOut + I.n0, shift(g.nodeSegOut, I.m0).data(), n, st);
  put<int>(d.nsIn + I.n0, shift(g.nodeSegIn, I.m0).data(), n, st);
  put<int>(d.segI0 + I.m0, shift(g.segI0, I.n0).data(), m, st);
  put<int>(d.segI1 + I.m0, shift(g.segI1, I.n0).data(), m, st);
  put<int>(d.jA + I.m0, shift(g.segJointA, I.p0).data(), m, st);
  put<int>(d.jB + I.m0, shift(g.segJointB, I.p0).data(), m, st);
  put<int>(d.segStrand + I.m0, shift(g.segStrand, I.s0).data(), m, st);
  put<int>(d.segLocal + I.m0, g.segLocal.data(), m, st);
  put<R>(d.l0 + I.m0, g.l0.data(), m, st);
  {
    std::vector<double> il(m);
    for (size_t j = 0; j < m; j++) il[j] = 1.0 / g.l0[j];
    put<W>(d.il0 + I.m0, il.data(), m, st);
  }
  put<int>(d.jS0 + I.p0, shift(g.jSeg0, I.m0).data(), p, st);
  put<int>(d.jS1 + I.p0, shift(g.jSeg1, I.m0).data(), p, st);
  put<R>(d.jLen + I.p0, g.jLen.data(), p, st);
  for (int side = 0; side < 2; side++) {
    std::vector<int> so(K), nsg(K), no(K);
    std::vector<double> w(K), h(K), fc(K), e9(K), hs(K);
    for (size_t q = 0; q < K; q++) { so[q] = I.m0 + g.cxSegOff[2 * q + side]; nsg[q] = g.cxNseg[2 * q + side]; w[q] = g.wk[2 * q + side]; h[q] = g.hk[2 * q + side]; }
    for (size_t q = 0; q < K; q++) no[q] = I.n0 + g.cxNodeOff[2 * q + side];
    for (size_t q = 0; q < K; q++) { fc[q] = g.fc90[2 * q + side]; e9[q] = g.E90[2 * q + side]; hs[q] = g.Hs[2 * q + side]; }
    put<R>(d.fc90 + size_t(side) * d.ktot + I.k0, fc.data(), K, st);
    put<R>(d.E90 + size_t(side) * d.ktot + I.k0, e9.data(), K, st);
    put<R>(d.Hs + size_t(side) * d.ktot + I.k0, hs.data(), K, st);
    put<int>(d.cxSegOff + size_t(side) * d.ktot + I.k0, so.data(), K, st);
    put<int>(d.cxNseg + size_t(side) * d.ktot + I.k0, nsg.data(), K, st);
    put<int>(d.cxNodeOff + size_t(side) * d.ktot + I.k0, no.data(), K, st);
    put<R>(d.wk + size_t(side) * d.ktot + I.k0, w.data(), K, st);
    put<R>(d.hk + size_t(side) * d.ktot + I.k0, h.data(), K, st);
  }
  {
    std::vector<int> ss(2 * K), sp(2 * K);
    for (size_t q = 0; q < 2 * K; q++) { ss[q] = I.s0 + g.cxStrand[g.sideList[q]]; sp[q] = 2 * I.k0 + g.sidePos[q]; }
    put<int>(d.sStrand + 2 * size_t(I.k0), ss.data(), 2 * K, st);
    put<int>(d.sPos + 2 * size_t(I.k0), sp.data(), 2 * K, st);
  }
  put<R>(d.cw + I.k0, g.w.data(), K, st);
  put<R>(d.ch + I.k0, g.h.data(), K, st);
  std::vector<int> so(S), sc(S);
  for (size_t s = 0; s < S; s++) { so[s] = 2 * I.k0 + g.strandSideOff[s]; sc[s] = g.strandSideCnt[s]; }
  put<int>(d.stSideOff + I.s0, so.data(), S, st);
  put<int>(d.stSideCnt + I.s0, sc.data(), S, st);
  std::vector<int> sg(S, 0);
  for (size_t q = 0; q < 2 * K; q++) sg[g.cxStrand[q]] = I.m0 + g.cxSegOff[q];
  put<int>(d.stSegOff + I.s0, sg.data(), S, st);
  std::vector<uint8_t> one(K, 1);
  put<uint8_t>(d.stuck + I.k0, one.data(), K, st);
  put<double>(d.utmSched + size_t(I.utmIdx) * WS_PROTOCOL_MAX_INC, g.proto.sched, WS_PROTOCOL_MAX_INC, st);
  const InstExt u = protocolState(g);
  put<InstExt>(d.ext + I.utmIdx, &u, 1, st);
  floorSections<P>(c, b);
  {
    // the joint and the clamp at every node, for the segment moments of the results (buildResults)
    std::vector<int> nj(n, -1), nc(n, -1);
    for (size_t j = 0; j < p; j++) nj[g.segI1[g.jSeg0[j]]] = I.p0 + int(j);
    for (size_t q = 0; q < g.cNode.size(); q++) nc[g.cNode[q]] = I.c0 + int(q);
    put<int>(d.nodeJoint + I.n0, nj.data(), n, st);
    put<int>(d.nodeClamp + I.n0, nc.data(), n, st);
  }
  displacementOrigin<P>(c, b);
}

// the ground's stick points of instance b start under its nodes as the host goals hold them
template <int P>
void floorStart(ws_ctx *c, int b) {
  Dev<P> &d = devOf<P>(c);
  using W = typename Dev<P>::W;
  const HostGoals &g = c->g[b];
  const InstDesc &I = c->inst[b];
  if (!g.prm.floor) return;
  std::vector<double> ax(g.n), ay(g.n);
  for (int i = 0; i < g.n; i++) { ax[i] = g.X[3 * size_t(i)]; ay[i] = g.X[3 * size_t(i) + 1]; }
  put<W>(d.flAx + I.n0, ax.data(), g.n, c->st);
  put<W>(d.flAy + I.n0, ay.data(), g.n, c->st);
}

// the contact-extension state of instance b at its start: no multiplier, no seats (wall slopes 1), no W2 reference angle
template <int P>
void resetExt(ws_ctx *c, int b) {
  Dev<P> &d = devOf<P>(c);
  using R = typename Dev<P>::R; using A = typename Dev<P>::A;
  const InstDesc &I = c->inst[b];
  const size_t K = I.K;
  if (!K) return;
  const std::vector<double> z(2 * K, 0.0), one(2 * K, 1.0), nan(K, std::numeric_limits<double>::quiet_NaN());
  put<A>(d.lam + I.k0, z.data(), K, c->st);
  put<A>(d.penAcc + I.k0, z.data(), K, c->st);
  put<R>(d.dent + 2 * size_t(I.k0), z.data(), 2 * K, c->st);
  put<R>(d.climb + 2 * size_t(I.k0), z.data(), 2 * K, c->st);
  put<R>(d.tanpsi + 2 * size_t(I.k0), one.data(), 2 * K, c->st);
  put<R>(d.dentE + I.k0, z.data(), K, c->st);
  put<R>(d.theta0 + I.k0, nan.data(), K, c->st);
  put<R>(d.Mrot + I.k0, z.data(), K, c->st);
  put<A>(d.rotSlip + I.k0, z.data(), K, c->st);
}

// the multiplier update of instance b that fell due at the end of its last iteration, applied before anything reads
// the multipliers or changes what the update depends on
template <int P>
void flushAL(ws_ctx *c, int b) {
  if (c->inst[b].aug && c->inst[b].contacts && c->inst[b].K) CK(launchAlFlush<P>(devOf<P>(c), c->dInst, c->dCtl, b, c->st));
}

template <int P>
void uploadAll(ws_ctx *c) {
  for (size_t b = 0; b < c->g.size(); b++) {
    resetExt<P>(c, int(b));
    uploadStatic<P>(c, int(b));
    floorStart<P>(c, int(b));
    uploadGoals<P>(c, int(b));
    uploadState<P>(c, int(b), 0, true);
    uploadState<P>(c, int(b), 1, false);
    uploadOrder<P>(c, int(b), 0);
    uploadOrder<P>(c, int(b), 1);
  }
  flushPuts(c);
}

// the short-slide side order holds when, in every instance with contacts, the slide limit (epsilon) is under half the
// shortest segment of the strands with crossings: a slide then moves a side by less than one segment per iteration
// (a segment would have to shorten by half to break it)
bool shortOrderOK(const ws_ctx *c) {
  if (c->sidesGeneral) return false;
  for (const HostGoals &g : c->g) {
    if (!g.K || !g.prm.contacts) continue;
    if (!(std::max(g.prm.epsilon, 1e-9) < 0.5 * g.sideSegMin())) return false;
  }
  return true;
}

template <int P>
void setupDev(ws_ctx *c) {
  Carver cnt{nullptr};
  Dev<P> &d = devOf<P>(c);
  layout<P>(d, cnt, c->z);
  c->bytes = cnt.off + 4096;
  CK(cudaMalloc(&c->arena, c->bytes));
  CK(cudaMemsetAsync(c->arena, 0, c->bytes, c->st));
  Carver cv{c->arena};
  layout<P>(d, cv, c->z);
  c->dExt = d.ext;
  uploadAll<P>(c);
}

// the earliest start of an instance in the last launch of the batched form (0: none recorded)
unsigned long long stepStart(const ws_ctx *c) {
  unsigned long long t0 = 0;
  for (size_t b = 0; b < c->ctlHost.size(); b++) {
    const InstCtl &s = c->ctlHost[b];
    if (b < c->ranLast.size() && !c->ranLast[b]) continue;     // left out of the last step by its mask
    if (s.tBeg && (!t0 || s.tBeg < t0)) t0 = s.tBeg;
  }
  return t0;
}

void readCtl(ws_ctx *c) {
  c->ctlHost.resize(c->inst.size());
  CK(cudaMemcpyAsync(c->ctlHost.data(), c->dCtl, sizeof(InstCtl) * c->inst.size(), cudaMemcpyDeviceToHost, c->st));
  c->extHost.assign(c->inst.size(), InstExt{});
  bool utm = false;
  for (const InstDesc &I : c->inst) utm = utm || I.utmMode || I.floorOn;
  if (utm && c->dExt) CK(cudaMemcpyAsync(c->extHost.data(), c->dExt, sizeof(InstExt) * c->inst.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
}
void fillControl(const InstCtl &s, const InstExt &u, ws_control *o, unsigned long long t0) {
  o->t_start_ms = (s.tBeg && t0 && s.tBeg >= t0) ? double(s.tBeg - t0) * 1e-6 : 0.0;
  o->t_end_ms = (s.tEnd && t0 && s.tEnd >= t0) ? double(s.tEnd - t0) * 1e-6 : 0.0;
  o->iter = s.iter; o->status = s.status; o->rollbacks = s.rollbacks; o->pending_zero = s.pending;
  o->ke = s.ke; o->ke_prev = s.ke_prev; o->residual = s.residual; o->res_force = s.res_f; o->res_torque = s.res_t; o->fref = s.fref;
  o->e_stretch = s.e_stretch; o->e_shear = s.e_shear; o->e_bend = s.e_bend; o->e_twist = s.e_twist; o->e_contact = s.e_contact;
  o->utm_inc = u.inc; o->utm_phase = u.phase; o->e_floor = u.eFloor;
}

// some instance runs an extension (contact extensions, the ground, a load protocol): the kernels' variants with them
bool anyExt(const ws_ctx *c) {
  for (const InstDesc &I : c->inst)
    if ((I.ext && I.contacts && I.K) || I.floorOn || I.utmMode) return true;
  return false;
}

#ifndef WSB_PLAIN_FORK
#define WSB_PLAIN_FORK 1     // the plain form's element phase as two kernels on forked branches (0: one kernel)
#endif
const PlainFork *plainFork(const ws_ctx *c) { return (WSB_PLAIN_FORK && c->fork.side) ? &c->fork : nullptr; }
// the plain form's launch mode when the options leave it to the environment: WEAVESIM_PLAIN_LAUNCH "roles" (one launch
// a phase, blocks in two roles), "serial" (one kernel a phase), else forked graph branches
int plainModeFromEnv() {
  const char *v = std::getenv("WEAVESIM_PLAIN_LAUNCH");
  if (v && std::strcmp(v, "roles") == 0) return 1;
  if (v && std::strcmp(v, "serial") == 0) return 2;
  return 0;
}
const PlainFork *plainForkOf(const ws_ctx *c) { return c->plainMode == 2 ? nullptr : plainFork(c); }

template <int P>
void stepImpl(ws_ctx *c, int nIter, const uint8_t *mask) {
  const int nInst = int(c->inst.size());
  const bool ext = anyExt(c);
  c->lastLaunches = 0;
  CK(cudaEventRecord(c->ev0, c->st));
  c->ranLast.assign(mask ? mask : nullptr, mask ? mask + nInst : nullptr);
  if (!mask) c->ranLast.assign(nInst, 1);
  if (c->form == WS_FORM_CTA) {
    if (mask) CK(cudaMemcpyAsync(c->dMask, mask, nInst, cudaMemcpyHostToDevice, c->st));
    const uint8_t *dm = mask ? c->dMask : nullptr;
    // the wide instances' clusters first on the context's stream, the one-block kernels beside them on a second
    // stream, joined before the step's end event
    cudaStream_t nst = c->st;
    if (c->nWide > 0 && nIter > 0) {
      CK(cudaEventRecord(c->ctaFork, c->st));
      CK(cudaStreamWaitEvent(c->sideCta, c->ctaFork, 0));
      CK(launchWide<P>(devOf<P>(c), c->dInst, c->dCtl, c->dWide, c->nWide, nIter, dm, 512, c->wideCl, c->shortSides, ext, c->st));
      nst = c->sideCta;
      c->lastLaunches += 1;
    }
    if (c->nNarrow > 0) {
      if (c->residentBytes) {
        const int thr = c->threads > 0 ? std::min(c->threads, 512) : 512;
        CK(launchResident<P>(devOf<P>(c), c->dInst, c->dCtl, c->dOrder, c->nNarrow, nIter, dm, thr, c->residentBytes,
                             c->shortSides, ext, nst));
      } else {
        const int thr = c->threads > 0 ? c->threads : 256;
        CK(launchBatched<P>(devOf<P>(c), c->dInst, c->dCtl, c->dOrder, c->nNarrow, nIter, dm, thr, c->nNarrow,
                            c->shortSides, ext, nst));
      }
      c->lastLaunches += 1;
    }
    if (nst != c->st) {
      CK(cudaEventRecord(c->ctaJoin, nst));
      CK(cudaStreamWaitEvent(c->st, c->ctaJoin, 0));
    }
  } else if (c->form == WS_FORM_GRID) {
    CK(cudaMemsetAsync(c->dBar, 0, 2 * sizeof(unsigned), c->st));
    CK(cudaMemsetAsync(c->dErr, 0, sizeof(int), c->st));
    if (nIter > 0)
      CK(launchGrid<P>(devOf<P>(c), c->dInst, c->dCtl, c->dPart, c->dBar, c->dErr, nIter, c->gridBlocks[c->shortSides][ext],
                       c->shortSides, ext, c->st));
    c->lastLaunches = 1;
  } else {
    const bool cx = c->inst[0].contacts && c->inst[0].K;
    const bool sh = c->shortSides;
    const int chunk = std::min(nIter, 50);
    const bool rb = c->inst[0].rbOn != 0;
    const int key = ((((chunk * 4 + c->plainMode) << 1) | (rb ? 1 : 0)) << 3) | (ext ? 4 : 0) | (cx ? 2 : 0) | (sh ? 1 : 0);
    if (chunk > 0 && (!c->graph || c->graphKey != key)) {
      if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
      cudaGraph_t gr;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      int nl = 0;
      for (int i = 0; i < chunk; i++)
        CK(launchPlainIter<P>(devOf<P>(c), c->dInst, c->dCtl, c->dPart, c->shape, cx, sh, ext, c->st, &nl, c->dBar + 2,
                              plainForkOf(c), c->plainMode == 1, rb));
      CK(cudaStreamEndCapture(c->st, &gr));
      CK(cudaGraphInstantiate(&c->graph, gr, 0));
      cudaGraphDestroy(gr);
      c->graphIters = chunk;
      c->graphKey = key;
      c->graphLaunches = nl;
    }
    int done = 0;
    while (nIter - done >= chunk && chunk > 0) { CK(cudaGraphLaunch(c->graph, c->st)); done += chunk; c->lastLaunches += c->graphLaunches; }
    int nl = 0;
    for (; done < nIter; done++)
      CK(launchPlainIter<P>(devOf<P>(c), c->dInst, c->dCtl, c->dPart, c->shape, cx, sh, ext, c->st, &nl, c->dBar + 2,
                            plainForkOf(c), c->plainMode == 1, rb));
    c->lastLaunches += nl;
  }
  CK(cudaEventRecord(c->ev1, c->st));
  if (c->form == WS_FORM_GRID) {
    int err = 0;
    CK(cudaMemcpyAsync(&err, c->dErr, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (err) throw std::runtime_error("grid barrier wait exceeded its limit; the step was abandoned");
  }
}

// the W1 classification is computed on the device when a download asks for any of its outputs
bool wantsClass(const ws_state_out *o) { return o->ctype || o->theta || o->phi || o->area || o->pressure || o->util; }

// download through the device: the requested fields are packed on the GPU in the caller's interleaved layout (the
// buffer selection and the roll-back flag read there), copied in one piece and split into the caller's arrays
template <int P>
void downloadPacked(ws_ctx *c, int b, ws_state_out *o) {
  const InstDesc &I = c->inst[b];
  PackList L{};
  size_t off = 0, elems = 0;
  struct Dst { void *p; size_t off, bytes; };
  std::vector<Dst> dst;
  auto add = [&](int kind, int count, int ncomp, void *p, bool bytes1) {
    if (!p || count <= 0) return;
    PackField &F = L.f[L.nf++];
    F.kind = kind; F.count = count; F.ncomp = ncomp; F.off = (long long)off;
    const size_t by = size_t(count) * ncomp * (bytes1 ? 1 : sizeof(double));
    dst.push_back({p, off, by});
    off += (by + 15) & ~size_t(15);
    elems = std::max(elems, size_t(count) * ncomp);
  };
  add(PF_X, I.n, 3, o->X, false); add(PF_Q, I.m, 4, o->Q, false); add(PF_V, I.n, 3, o->V, false);
  add(PF_W, I.m, 3, o->W, false); add(PF_U, I.K, 2, o->u, false); add(PF_NPREV, I.K, 3, o->nprev, false);
  add(PF_SLIP, I.K, 1, o->slip, false); add(PF_FN, I.K, 1, o->Fn, false); add(PF_FT, I.K, 1, o->Ft, false);
  add(PF_GAP, I.K, 1, o->gap, false); add(PF_N, I.m, 1, o->N, false); add(PF_VSH, I.m, 2, o->Vsh, false);
  add(PF_M, I.p, 3, o->M, false); add(PF_REACT, I.n, 3, o->reactions, false);
  add(PF_STUCK, I.K, 1, o->stuck, true); add(PF_STATE, I.K, 1, o->state, true);
  add(PF_CTYPE, I.K, 1, o->ctype, true); add(PF_THETA, I.K, 1, o->theta, false); add(PF_PHI, I.K, 2, o->phi, false);
  add(PF_AREA, I.K, 1, o->area, false); add(PF_PRES, I.K, 1, o->pressure, false); add(PF_UTIL, I.K, 1, o->util, false);
  add(PF_LAM, I.K, 1, o->lambda, false); add(PF_DENT, I.K, 1, o->dent, false); add(PF_MROT, I.K, 1, o->M_rot, false);
  add(PF_RSLIP, I.K, 1, o->rot_slip, false);
  add(PF_UTM, WS_PROTOCOL_MAX_INC, 4, o->utm, false);
  add(PF_FLF, I.n, 3, o->floor_F, false); add(PF_FLS, I.n, 1, o->floor_state, true);
  add(PF_SEGM, I.m, 3, o->seg_M, false); add(PF_NODEM, I.n, 4, o->node_M, false); add(PF_DISP, I.n, 3, o->disp, false);
  if (!L.nf) return;
  if (o->lambda) flushAL<P>(c, b);
  if (o->seg_M || o->node_M) CK(launchResults<P>(devOf<P>(c), c->dInst, b, I.n, I.m, c->st));
  if (wantsClass(o)) CK(launchClassify<P>(devOf<P>(c), c->dInst, b, I.K, c->st));
  unsigned char *dv = xferBuf(c, off);
  CK(launchPack<P>(devOf<P>(c), c->dInst, c->dCtl, b, L, elems, dv, c->st));
  char *h = stageBuf(c, off);
  std::vector<Piece> ps;
  for (const Dst &q : dst) ps.push_back({static_cast<char *>(q.p), q.off, q.bytes});
  const int nc = chunkCount(off);
  for (int k = 0; k < nc; k++) {
    const size_t a = chunkEdge(off, nc, k), e = chunkEdge(off, nc, k + 1);
    if (e > a) CK(cudaMemcpyAsync(h + a, dv + a, e - a, cudaMemcpyDeviceToHost, c->st));
    CK(cudaEventRecord(c->evChunk[k], c->st));
  }
  for (int k = 0; k < nc; k++) {
    CK(cudaEventSynchronize(c->evChunk[k]));
    copyRange(ps, h, chunkEdge(off, nc, k), chunkEdge(off, nc, k + 1), false);
  }
}

template <int P>
void downloadImpl(ws_ctx *c, int b, ws_state_out *o) {
  if (c->pinnedOK) { downloadPacked<P>(c, b, o); return; }
  Dev<P> &d = devOf<P>(c);
  if (o->lambda) flushAL<P>(c, b);
  readCtl(c);
  const InstCtl &s = c->ctlHost[b];
  const InstDesc &I = c->inst[b];
  const size_t n = I.n, m = I.m, p = I.p, K = I.K;
  Fetch f;
  if (o->X) f.pairs(d.X + size_t(s.cur * 3) * d.ntot, PrecT<P>::TWO ? d.Xlo + size_t(s.cur * 3) * d.ntot : nullptr, d.ntot, I.n0, n, 3, o->X);
  if (o->Q) f.pairs(d.Q + size_t(s.cur * 4) * d.mtot, PrecT<P>::TWO ? d.Qlo + size_t(s.cur * 4) * d.mtot : nullptr, d.mtot, I.m0, m, 4, o->Q);
  if (o->V) { if (s.pending) std::fill(o->V, o->V + 3 * n, 0.0); else f.planes(d.V, d.ntot, I.n0, n, 3, o->V); }
  if (o->W) { if (s.pending) std::fill(o->W, o->W + 3 * m, 0.0); else f.planes(d.Wr, d.mtot, I.m0, m, 3, o->W); }
  if (K) {
    if (o->u) f.planes(d.u, d.ktot, I.k0, K, 2, o->u);
    if (o->nprev) f.planes(d.nPrev, d.ktot, I.k0, K, 3, o->nprev);
    if (o->slip) f.planes(d.slip, 0, I.k0, K, 1, o->slip);
    if (o->Fn) f.planes(d.Fn, 0, I.k0, K, 1, o->Fn);
    if (o->Ft) f.planes(d.Ft, 0, I.k0, K, 1, o->Ft);
    if (o->gap) f.planes(d.gap, 0, I.k0, K, 1, o->gap);
    if (o->stuck) f.bytes(d.stuck + I.k0, K, o->stuck);
    if (o->state) f.bytes(d.cstate + I.k0, K, o->state);
    if (wantsClass(o)) {
      CK(launchClassify<P>(d, c->dInst, b, I.K, c->st));
      if (o->ctype) f.bytes(d.ctype + I.k0, K, o->ctype);
      if (o->theta) f.planes(d.theta, 0, I.k0, K, 1, o->theta);
      if (o->phi) f.planes(d.phiS, 0, 2 * size_t(I.k0), 2 * K, 1, o->phi);
      if (o->area) f.planes(d.area, 0, I.k0, K, 1, o->area);
      if (o->pressure) f.planes(d.pres, 0, I.k0, K, 1, o->pressure);
      if (o->util) f.planes(d.util, 0, I.k0, K, 1, o->util);
    }
    if (o->lambda) f.planes(d.lam, 0, I.k0, K, 1, o->lambda);
    if (o->M_rot) f.planes(d.Mrot, 0, I.k0, K, 1, o->M_rot);
    if (o->rot_slip) f.planes(d.rotSlip, 0, I.k0, K, 1, o->rot_slip);
    if (o->dent) {
      double *dd = f.scratch(2 * K), *de = f.scratch(K);
      f.planes(d.dent, 0, 2 * size_t(I.k0), 2 * K, 1, dd);
      f.planes(d.dentE, 0, I.k0, K, 1, de);
      f.after.push_back([dd, de, K, out = o->dent]() {
        for (size_t q = 0; q < K; q++) out[q] = dd[2 * q] + dd[2 * q + 1] + de[q];
      });
    }
  }
  if (o->N) f.planes(d.Nax, 0, I.m0, m, 1, o->N);
  if (o->Vsh) f.planes(d.Vsh, d.mtot, I.m0, m, 2, o->Vsh);
  if (o->M && p) f.planes(d.Mj, d.ptot, I.p0, p, 3, o->M);
  if (o->reactions) f.planes(d.react, d.ntot, I.n0, n, 3, o->reactions);
  if (o->utm) f.planes(d.utmOut, 0, size_t(I.utmIdx) * 4 * WS_PROTOCOL_MAX_INC, 4 * WS_PROTOCOL_MAX_INC, 1, o->utm);
  if (o->floor_F) f.planes(d.flF, d.ntot, I.n0, n, 3, o->floor_F);
  if (o->floor_state) f.bytes(d.flState + I.n0, n, o->floor_state);
  if (o->seg_M || o->node_M) CK(launchResults<P>(d, c->dInst, b, I.n, I.m, c->st));
  if (o->seg_M) f.planes(d.segM, d.mtot, I.m0, m, 3, o->seg_M);
  if (o->node_M) f.planes(d.nodeLay, d.ntot, I.n0, n, 4, o->node_M);
  if (o->disp) {
    double *x = f.scratch(3 * n), *x0 = f.scratch(3 * n);
    f.pairs(d.X + size_t(s.cur * 3) * d.ntot, PrecT<P>::TWO ? d.Xlo + size_t(s.cur * 3) * d.ntot : nullptr, d.ntot, I.n0, n, 3, x);
    f.planes(d.X0, d.ntot, I.n0, n, 3, x0);
    f.after.push_back([x, x0, n, out = o->disp]() { for (size_t q = 0; q < 3 * n; q++) out[q] = x[q] - x0[q]; });
  }
  f.run(c);
}

// current X, Q, u, nPrev of instance b into its host goals
template <int P>
void pullState(ws_ctx *c, int b) {
  HostGoals &g = c->g[b];
  ws_state_out o{};
  std::vector<double> X(3 * size_t(g.n)), Q(4 * size_t(g.m)), u(2 * size_t(g.K)), np(3 * size_t(g.K));
  o.X = X.data(); o.Q = Q.data();
  if (g.K) { o.u = u.data(); o.nprev = np.data(); }
  downloadImpl<P>(c, b, &o);
  g.X = X; g.Q = Q;
  if (g.K) { g.u = u; g.nPrev = np; }
}

// the batched form keeps its instances in shared memory when the largest fits a block (re-evaluated when the side
// order changes, as the layout depends on it)
template <int P>
void selectResident(ws_ctx *c) {
  c->residentBytes = 0;
  if (c->form != WS_FORM_CTA || c->ctaGlobal) return;
  for (const InstDesc &I : c->inst)
    if (I.rbOn) return;          // the rigid-body freedoms step from the iteration's start, which global state keeps
  size_t need = 0;
  for (size_t b = 0; b < c->inst.size(); b++) {
    if (c->isWide[b]) continue;                 // the wide instances run with global state in the cluster kernel
    const InstDesc &I = c->inst[b];
    need = std::max<size_t>(need, residentLayout<P>(I.n, I.m, I.p, I.C, I.K, c->shortSides).bytes);
  }
  size_t granted = 0;
  CK(residentPrepare<P>(need, c->shortSides, &granted));
  c->residentBytes = granted;
}

// clusters of `cl` blocks of 512 threads that the device can hold at once, for the cluster kernel's variants that need
// the most resources (0: the shape cannot launch)
int wideFit(int prec, int cl) {
  int fit = 1 << 30;
  for (int sh = 0; sh < 2; sh++)
    for (int ex = 0; ex < 2; ex++) {
      int n = 0;
      switch (prec) {
        case WS_PREC_F64: n = wideClusters<PREC_F64>(512, cl, sh != 0, ex != 0); break;
        case WS_PREC_MIXED: n = wideClusters<PREC_MIXED>(512, cl, sh != 0, ex != 0); break;
        default: n = wideClusters<PREC_F32>(512, cl, sh != 0, ex != 0); break;
      }
      fit = std::min(fit, n);
    }
  return fit;
}

// the launch shape `sh` (the batched form's block size, state placement and wide instances; the plain form's launch
// mode): an instance is wide from sh.wide_min nodes + segments up (never with a load protocol), so its width depends on
// its own size and the shape only, never on the rest of the batch
template <int P>
void applyShape(ws_ctx *c, const ws_shape &sh) {
  c->launch = sh;
  c->launch.source = 0;
  c->threads = sh.threads;
  c->ctaGlobal = sh.cta_state == WS_CTA_GLOBAL;
  c->plainMode = sh.plain_launch;
  c->wideCl = c->form == WS_FORM_CTA ? sh.wide_cluster : 1;
  c->wideMin = sh.wide_min > 0 ? sh.wide_min : 32768;
  // a cluster shape the device cannot hold is halved until it can (1: no wide instances)
  while (c->wideCl >= 2 && wideFit(c->prec, c->wideCl) == 0) c->wideCl /= 2;
  const int nInst = int(c->inst.size());
  c->isWide.assign(nInst, 0);
  std::vector<int> wide, narrow;
  for (int b : c->order) {
    const InstDesc &I = c->inst[b];
    const bool w = c->form == WS_FORM_CTA && c->wideCl >= 2 && I.n + I.m >= c->wideMin && !I.utmMode && !I.rbOn;
    c->isWide[b] = w;
    (w ? wide : narrow).push_back(b);
  }
  c->nWide = int(wide.size());
  c->nNarrow = int(narrow.size());
  if (c->nWide == 0) c->wideCl = 0;
  c->launch.wide_cluster = c->wideCl ? c->wideCl : 1;
  if (c->nNarrow) CK(cudaMemcpyAsync(c->dOrder, narrow.data(), sizeof(int) * c->nNarrow, cudaMemcpyHostToDevice, c->st));
  if (c->nWide) CK(cudaMemcpyAsync(c->dWide, wide.data(), sizeof(int) * c->nWide, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));    // the host vectors above go out of scope
  selectResident<P>(c);
}

// what the choice of shape depends on, for the tuner's size bucket
TuneInfo tuneInfo(const ws_ctx *c) {
  TuneInfo t;
  t.form = c->form; t.prec = c->prec; t.nInst = int(c->inst.size()); t.shortSides = c->shortSides ? 1 : 0; t.ext = anyExt(c);
  for (const InstDesc &I : c->inst) {
    t.maxElems = std::max<long long>(t.maxElems, I.n + I.m);
    t.totalElems += I.n + I.m;
  }
  return t;
}
std::string deviceName(int dev) {
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) { cudaGetLastError(); return "none"; }
  return std::string(p.name) + "-sm" + std::to_string(p.multiProcessorCount);
}

// The autotuner: every candidate shape (tune.cpp) runs the same short trial from the context's starting state, timed with
// CUDA events on the context's stream after an untimed run of the same length (for the plain form, the graph capture);
// the fastest is kept, stored in the cache under the batch's size bucket, and the starting state is put back.  The
// state is restored between trials from a device copy of the arena and the control blocks (or, when the device has no
// room for the copy, by uploading the starting state again from the host goals).
template <int P>
void tuneCtx(ws_ctx *c) {
  const TuneInfo info = tuneInfo(c);
  const std::string key = tuneKey(deviceName(c->device), info);
  ws_shape hit{};
  if (tuneLookup(key, &hit)) {
    applyShape<P>(c, hit);
    c->launch = hit;
    c->launch.wide_cluster = c->wideCl ? c->wideCl : 1;
    c->launch.source = 2;
    return;
  }
  const int nInst = int(c->inst.size());
  std::vector<InstCtl> ctl0(nInst);
  CK(cudaMemcpyAsync(ctl0.data(), c->dCtl, sizeof(InstCtl) * nInst, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  char *snap = nullptr;
  size_t freeB = 0, totalB = 0;
  if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess && freeB > c->bytes + (size_t(1) << 30)) {
    if (cudaMalloc(&snap, c->bytes) != cudaSuccess) { cudaGetLastError(); snap = nullptr; }
  }
  if (snap) CK(cudaMemcpyAsync(snap, c->arena, c->bytes, cudaMemcpyDeviceToDevice, c->st));
  auto restore = [&]() {
    if (snap) {
      CK(cudaMemcpyAsync(c->arena, snap, c->bytes, cudaMemcpyDeviceToDevice, c->st));
    } else {
      CK(cudaMemsetAsync(c->arena, 0, c->bytes, c->st));
      uploadAll<P>(c);
    }
    CK(cudaMemcpyAsync(c->dCtl, ctl0.data(), sizeof(InstCtl) * nInst, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
  };
  const int iters = c->form == WS_FORM_PLAIN ? 200 : 50;
  auto trial = [&](const ws_shape &sh) {
    applyShape<P>(c, sh);
    restore();
    stepImpl<P>(c, iters, nullptr);      // untimed: first launches, graph capture
    restore();
    stepImpl<P>(c, iters, nullptr);
    float ms = 0;
    CK(cudaEventSynchronize(c->ev1));
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    return double(ms);
  };
  // shapes that launch the same kernels the same way are timed once
  auto effective = [&]() {
    return std::to_string(c->form == WS_FORM_CTA ? (c->threads > 0 ? c->threads : (c->residentBytes ? 512 : 256)) : 0) + "/" +
           std::to_string(c->residentBytes ? 1 : 0) + "/" + std::to_string(c->wideCl) + "/" + std::to_string(c->nWide) + "/" +
           std::to_string(c->plainMode);
  };
  std::map<std::string, double> seen;
  ws_shape best{};
  double bestMs = INFINITY, defMs = NAN;
  int trials = 0;
  auto run = [&](const std::vector<ws_shape> &cands) {
    for (const ws_shape &sh : cands) {
      applyShape<P>(c, sh);
      const std::string e = effective();
      double ms;
      auto it = seen.find(e);
      if (it != seen.end()) {
        ms = it->second;
      } else {
        ms = trial(sh);
        seen[e] = ms;
        trials++;
      }
      if (ms < bestMs) { bestMs = ms; best = sh; }
    }
  };
  // the default shape first, for comparison
  ws_shape def{};
  def.threads = 0; def.cta_state = WS_CTA_AUTO; def.wide_cluster = 2; def.wide_min = 32768; def.plain_launch = 0;
  run({def});
  defMs = bestMs;
  run(tuneStage1(info));
  run(tuneStage2(info, best));
  applyShape<P>(c, best);
  restore();
  if (snap) cudaFree(snap);
  // the plain form's graph of the trial length is kept; a step of another length captures its own
  c->launch.source = 1;
  c->launch.trials = trials;
  c->launch.trial_ms = bestMs;
  c->launch.default_ms = defMs;
  tuneStore(key, c->launch);
}

// a warm start may change the slide limit or switch contacts: on a change of side order, every instance's order and
// keys are rebuilt from its current slide coordinates into the buffer its next iteration reads
template <int P>
void reselectOrder(ws_ctx *c) {
  const bool ok = shortOrderOK(c);
  if (ok == c->shortSides) return;
  readCtl(c);
  for (size_t b = 0; b < c->g.size(); b++) {
    pullState<P>(c, int(b));
    c->g[b].sortSides();
    uploadOrder<P>(c, int(b), c->ctlHost[b].obuf);
  }
  flushPuts(c);
  c->shortSides = ok;
  selectResident<P>(c);
}

template <int P>
void setParamsImpl(ws_ctx *c, int b, const ws_model *md) {
  flushAL<P>(c, b);
  pullState<P>(c, b);
  HostGoals &g = c->g[b];
  const std::vector<int> oldSeg = g.cSeg;
  const bool hadFloor = g.prm.floor != 0;
  HostGoals trial = g;
  trial.rebuild(*md);
  if (trial.cSeg != oldSeg) throw std::invalid_argument("the anchors changed the rotation clamps: create a new context");
  g = std::move(trial);
  Sizes off;
  off.n = c->inst[b].n0; off.m = c->inst[b].m0; off.p = c->inst[b].p0; off.c = c->inst[b].c0; off.k = c->inst[b].k0; off.s = c->inst[b].s0;
  off.b = b;
  c->inst[b] = describe(g, off);
  CK(cudaMemcpyAsync(c->dInst + b, &c->inst[b], sizeof(InstDesc), cudaMemcpyHostToDevice, c->st));
  uploadGoals<P>(c, b);
  floorSections<P>(c, b);     // the ground's sections may have changed
  if (!hadFloor) floorStart<P>(c, b);     // a new ground starts its stick points under the nodes (solver_cpu.js:689-690)
  flushPuts(c);
  readCtl(c);
  InstCtl s = c->ctlHost[b];
  s.ke_prev = 0.0; s.status = WS_RUNNING; s.disp_it0 = s.iter;
  // a rebuild restarts the multipliers' penetration window (solver_cpu.js:688)
  s.penN = 0; s.alPend = 0;
  {
    using A = typename Dev<P>::A;
    if (g.K) CK(cudaMemsetAsync(devOf<P>(c).penAcc + c->inst[b].k0, 0, sizeof(A) * g.K, c->st));
  }
  CK(cudaMemcpyAsync(c->dCtl + b, &s, sizeof(InstCtl), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  reselectOrder<P>(c);
}

template <int P>
void loadInstanceImpl(ws_ctx *c, int b, const ws_model *md) {
  HostGoals g;
  g.build(*md);
  const HostGoals &o = c->g[b];
  if (g.n != o.n || g.m != o.m || g.p != o.p || g.K != o.K || g.S != o.S || g.C != o.C)
    throw std::invalid_argument("the model's element counts differ from the slot's");
  if (c->form == WS_FORM_GRID && g.proto.mode)
    throw std::invalid_argument("a load protocol runs in the cta and plain forms, not the grid form");
  c->g[b] = std::move(g);
  Sizes off;
  off.n = c->inst[b].n0; off.m = c->inst[b].m0; off.p = c->inst[b].p0; off.c = c->inst[b].c0; off.k = c->inst[b].k0; off.s = c->inst[b].s0;
  off.b = b;
  c->inst[b] = describe(c->g[b], off);
  CK(cudaMemcpyAsync(c->dInst + b, &c->inst[b], sizeof(InstDesc), cudaMemcpyHostToDevice, c->st));
  uploadStatic<P>(c, b);
  uploadGoals<P>(c, b);
  floorStart<P>(c, b);
  Dev<P> &d = devOf<P>(c);
  using A = typename Dev<P>::A;
  if (o.K) CK(cudaMemsetAsync(d.slip + c->inst[b].k0, 0, sizeof(A) * o.K, c->st));
  using R = typename Dev<P>::R;
  for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(d.react + size_t(k) * d.ntot + c->inst[b].n0, 0, sizeof(R) * o.n, c->st));
  InstCtl s;
  std::memset(&s, 0, sizeof(s));
  s.status = WS_RUNNING; s.residual = INFINITY;
  resetExt<P>(c, b);
  uploadState<P>(c, b, 0, true);
  // both buffers: a slice left over from the slot's previous model could point into another strand's sides
  uploadOrder<P>(c, b, 0);
  uploadOrder<P>(c, b, 1);
  flushPuts(c);
  CK(cudaMemcpyAsync(c->dCtl + b, &s, sizeof(InstCtl), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  reselectOrder<P>(c);
}

// upload through the device: the caller's arrays go up as they are, one copy, and the GPU splits them into planes,
// clears the velocities, resets the control block and (with u) rebuilds the side order from the new slide coordinates.
// The host goals keep their older copy of the state; every consumer of it pulls the current state first.
template <int P>
void uploadStatePacked(ws_ctx *c, int b, const double *X, const double *Q, const double *u) {
  const InstDesc &I = c->inst[b];
  const size_t nX = 3 * size_t(I.n), nQ = 4 * size_t(I.m), nU = (u && I.K) ? 2 * size_t(I.K) : 0;
  const size_t bytes = (nX + nQ + nU) * sizeof(double);
  char *h = stageBuf(c, bytes);
  unsigned char *dv = xferBuf(c, bytes);
  const std::vector<Piece> ps = {{(char *)X, 0, nX * sizeof(double)}, {(char *)Q, nX * sizeof(double), nQ * sizeof(double)},
                                 {(char *)u, (nX + nQ) * sizeof(double), nU * sizeof(double)}};
  const int nc = chunkCount(bytes);
  for (int k = 0; k < nc; k++) {
    const size_t a = chunkEdge(bytes, nc, k), e = chunkEdge(bytes, nc, k + 1);
    if (e <= a) continue;
    copyRange(ps, h, a, e, true);
    CK(cudaMemcpyAsync(dv + a, h + a, e - a, cudaMemcpyHostToDevice, c->st));
  }
  CK(launchUnpack<P>(devOf<P>(c), c->dInst, c->dCtl, b, reinterpret_cast<const double *>(dv), I.n, I.m, I.K, nU > 0, true,
                     c->shortSides, c->st));
  CK(cudaStreamSynchronize(c->st));
}

template <int P>
void uploadStateImpl(ws_ctx *c, int b, const double *X, const double *Q, const double *u) {
  flushAL<P>(c, b);
  if (c->pinnedOK) { uploadStatePacked<P>(c, b, X, Q, u); return; }
  HostGoals &g = c->g[b];
  readCtl(c);
  InstCtl s = c->ctlHost[b];
  g.X.assign(X, X + 3 * size_t(g.n));
  g.Q.assign(Q, Q + 4 * size_t(g.m));
  if (u && g.K) g.u.assign(u, u + 2 * size_t(g.K));
  g.startProtocol();          // an upload restarts the load protocol from the uploaded probe (solver_gpu.js:286,296-311)
  uploadState<P>(c, b, s.cur, u != nullptr);
  floorStart<P>(c, b);
  if (g.proto.mode) {
    const InstExt pu = protocolState(g);
    put<InstExt>(devOf<P>(c).ext + c->inst[b].utmIdx, &pu, 1, c->st);
  }
  flushPuts(c);
  if (u && g.K) { g.sortSides(); uploadOrder<P>(c, b, s.obuf); flushPuts(c); }
  s.pending = 0; s.ke_prev = 0.0; s.status = WS_RUNNING;
  CK(cudaMemcpyAsync(c->dCtl + b, &s, sizeof(InstCtl), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
}

template <int P>
void internalizeImpl(ws_ctx *c, int b) {
  pullState<P>(c, b);
  HostGoals &g = c->g[b];
  g.X0 = g.X;
  displacementOrigin<P>(c, b);
  flushPuts(c);
  Dev<P> &d = devOf<P>(c);
  using A = typename Dev<P>::A;
  if (g.K) CK(cudaMemsetAsync(d.slip + c->inst[b].k0, 0, sizeof(A) * g.K, c->st));
  CK(cudaStreamSynchronize(c->st));
}

template <class F>
int guarded(const char *what, F &&f) {
  struct Drop { ~Drop() { dropPuts(); } } drop;     // nothing queued outlives the call, failed or not
  try {
    f();
    return WS_OK;
  } catch (const CudaError &e) {
    return fail(WS_ERR_CUDA, std::string(what) + ": " + e.what());
  } catch (const std::invalid_argument &e) {
    return fail(WS_ERR_ARG, std::string(what) + ": " + e.what());
  } catch (const std::bad_alloc &) {
    return fail(WS_ERR_NOMEM, std::string(what) + ": host memory exhausted");
  } catch (const std::exception &e) {
    return fail(WS_ERR_STATE, std::string(what) + ": " + e.what());
  }
}

#define DISPATCH(c, FN, ...)                                  \
  switch ((c)->prec) {                                        \
    case WS_PREC_F64: FN<PREC_F64>(__VA_ARGS__); break;       \
    case WS_PREC_MIXED: FN<PREC_MIXED>(__VA_ARGS__); break;   \
    default: FN<PREC_F32>(__VA_ARGS__); break;                \
  }

void destroyCtx(ws_ctx *c) {
  if (!c) return;
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->arena) cudaFree(c->arena);
  if (c->dInst) cudaFree(c->dInst);
  if (c->dCtl) cudaFree(c->dCtl);
  if (c->dOrder) cudaFree(c->dOrder);
  if (c->dWide) cudaFree(c->dWide);
  if (c->sideCta) cudaStreamDestroy(c->sideCta);
  if (c->ctaFork) cudaEventDestroy(c->ctaFork);
  if (c->ctaJoin) cudaEventDestroy(c->ctaJoin);
  if (c->dMask) cudaFree(c->dMask);
  if (c->dPart) cudaFree(c->dPart);
  if (c->dBar) cudaFree(c->dBar);
  if (c->dErr) cudaFree(c->dErr);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  for (cudaEvent_t e : c->evChunk)
    if (e) cudaEventDestroy(e);
  if (c->st) cudaStreamDestroy(c->st);
  if (c->fork.side) cudaStreamDestroy(c->fork.side);
  if (c->fork.fork) cudaEventDestroy(c->fork.fork);
  if (c->fork.join) cudaEventDestroy(c->fork.join);
  if (c->fork.fork2) cudaEventDestroy(c->fork.fork2);
  if (c->fork.join2) cudaEventDestroy(c->fork.join2);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->dXfer) cudaFree(c->dXfer);
  delete c;
}

}  // namespace

extern "C" {

int ws_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n;
}

int ws_create(const ws_model *const *models, int32_t n_instances, const ws_opts *opts, ws_ctx **out) {
  if (!models || n_instances <= 0 || !out) return fail(WS_ERR_ARG, "ws_create: need at least one model and an output pointer");
  ws_opts o{};
  if (opts) o = *opts;
  if (o.precision < 0 || o.precision > 2) return fail(WS_ERR_ARG, "ws_create: unknown precision");
  if (o.form < 0 || o.form > 2) return fail(WS_ERR_ARG, "ws_create: unknown execution form");
  if (o.form != WS_FORM_CTA && n_instances != 1) return fail(WS_ERR_ARG, "ws_create: the grid and plain forms take one instance");
  if (o.threads < 0 || o.threads > 512 || (o.threads % 32)) return fail(WS_ERR_ARG, "ws_create: threads must be a multiple of 32 up to 512");
  if (ws_device_count() <= 0) return fail(WS_ERR_NODEV, "ws_create: no CUDA device (this library has no CPU path)");
  auto c = new ws_ctx();
  c->prec = o.precision; c->form = o.form; c->threads = o.threads; c->device = o.device;
  if (o.side_order < 0 || o.side_order > 1) { delete c; return fail(WS_ERR_ARG, "ws_create: unknown side order"); }
  c->sidesGeneral = o.side_order == WS_SIDES_GENERAL;
  if (o.cta_state < 0 || o.cta_state > 1) { delete c; return fail(WS_ERR_ARG, "ws_create: unknown cta_state"); }
  c->ctaGlobal = o.cta_state == WS_CTA_GLOBAL;
  int rc = guarded("ws_create", [&]() {
    CK(cudaSetDevice(o.device));
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    if (o.form == WS_FORM_PLAIN) {
      CK(cudaStreamCreateWithFlags(&c->fork.side, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&c->fork.fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->fork.join, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->fork.fork2, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->fork.join2, cudaEventDisableTiming));
      c->plainMode = plainModeFromEnv();
    }
    c->pinnedOK = true;
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    for (cudaEvent_t &e : c->evChunk) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->g.resize(n_instances);
    Sizes off;
    for (int b = 0; b < n_instances; b++) {
      if (!models[b]) throw std::invalid_argument("null model");
      c->g[b].build(*models[b]);
      if (o.form == WS_FORM_GRID && c->g[b].proto.mode)
        throw std::invalid_argument("a load protocol runs in the cta and plain forms, not the grid form");
      if (o.form == WS_FORM_GRID && c->g[b].rigid)
        throw std::invalid_argument("a model that only the ground holds runs in the cta and plain forms, not the grid form");
      off.b = b;
      c->inst.push_back(describe(c->g[b], off));
      off.n += c->g[b].n; off.m += c->g[b].m; off.p += c->g[b].p; off.c += c->g[b].C; off.k += c->g[b].K; off.s += c->g[b].S;
    }
    c->z = off;
    c->z.b = n_instances;
    // longest instances first: the hardware block scheduler then balances the tail
    c->order.resize(n_instances);
    std::iota(c->order.begin(), c->order.end(), 0);
    std::stable_sort(c->order.begin(), c->order.end(), [&](int a, int b) { return c->inst[a].n + c->inst[a].m > c->inst[b].n + c->inst[b].m; });
    if (o.wide_cluster < 0 || o.wide_cluster > 8 || o.wide_min < 0)
      throw std::invalid_argument("wide_cluster must be 0 (default), 1 (off) or 2..8; wide_min 0 (default) or more");
    if (o.tune < 0 || o.tune > 1) throw std::invalid_argument("tune must be 0 or 1");
    CK(cudaMalloc(&c->dInst, sizeof(InstDesc) * n_instances));
    CK(cudaMalloc(&c->dCtl, sizeof(InstCtl) * n_instances));
    CK(cudaMalloc(&c->dOrder, sizeof(int) * n_instances));
    CK(cudaMalloc(&c->dWide, sizeof(int) * n_instances));
    CK(cudaMalloc(&c->dMask, n_instances));
    CK(cudaMemcpyAsync(c->dInst, c->inst.data(), sizeof(InstDesc) * n_instances, cudaMemcpyHostToDevice, c->st));
    if (o.form == WS_FORM_CTA) {
      CK(cudaStreamCreateWithFlags(&c->sideCta, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&c->ctaFork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->ctaJoin, cudaEventDisableTiming));
    }
    std::vector<InstCtl> ctl(n_instances);
    for (int b = 0; b < n_instances; b++) {
      InstCtl &s = ctl[b];
      std::memset(&s, 0, sizeof(s));
      s.status = WS_RUNNING; s.residual = INFINITY;
    }
    CK(cudaMemcpyAsync(c->dCtl, ctl.data(), sizeof(InstCtl) * n_instances, cudaMemcpyHostToDevice, c->st));
    const InstDesc &I0 = c->inst[0];
    auto blocks = [](long long cnt, int thr) { return int(std::max<long long>(1, std::min<long long>((cnt + thr - 1) / thr, 148LL * 8))); };
    c->shape.blocksA = blocks(I0.m + I0.p + I0.C + 2LL * I0.K, 256);
    c->shape.blocksDS = blocks(I0.n + I0.m + 2LL * I0.K, 256);
    c->shape.blocksX = blocks(2LL * I0.K, 128);
    c->shape.blocksXR = blocks(2LL * I0.K, 256);
    c->shape.blocksY = blocks(I0.m + I0.p + I0.C, 256);
    c->shape.pairsY = std::max(1, std::max(I0.m, I0.p + I0.C));
    c->shape.blocksDN = blocks(I0.n, 256);
    c->shape.blocksDNS = blocks(I0.n + 2LL * I0.K, 256);
    c->shape.blocksDM = blocks(I0.m, 256);
    c->shape.blocksR = blocks(I0.m + 2LL * I0.K, 256);
    c->shape.blocksD = blocks(I0.n + I0.m, 256);
    for (int sh = 0; sh < 2; sh++)
      for (int ex = 0; ex < 2; ex++) {
        switch (c->prec) {
          case WS_PREC_F64: c->gridBlocks[sh][ex] = gridBlocks<PREC_F64>(sh != 0, ex != 0); break;
          case WS_PREC_MIXED: c->gridBlocks[sh][ex] = gridBlocks<PREC_MIXED>(sh != 0, ex != 0); break;
          default: c->gridBlocks[sh][ex] = gridBlocks<PREC_F32>(sh != 0, ex != 0); break;
        }
      }
    CK(cudaGetLastError());
    const int parts = std::max({c->shape.blocksA + c->shape.blocksDS, c->shape.blocksA + c->shape.blocksD,
                                c->shape.blocksX + c->shape.blocksY + std::max(c->shape.blocksDN, c->shape.blocksDNS) + c->shape.blocksDM,
                                c->gridBlocks[0][0], c->gridBlocks[0][1], c->gridBlocks[1][0], c->gridBlocks[1][1]});
    // one row more than the blocks: the plain form's summary of the element and node partials
    CK(cudaMalloc(&c->dPart, sizeof(double) * (RS_NSUM + RX_NMAX) * (size_t(parts) + 1)));
    // [0..1] grid barrier; [2..3] the plain form's finishing-block counter (64 bits in the split update phase)
    CK(cudaMalloc(&c->dBar, 4 * sizeof(unsigned)));
    CK(cudaMemsetAsync(c->dBar, 0, 4 * sizeof(unsigned), c->st));
    CK(cudaMalloc(&c->dErr, sizeof(int)));
    c->shortSides = shortOrderOK(c);
    DISPATCH(c, setupDev, c);
    ws_shape sh{};
    sh.threads = o.threads; sh.cta_state = o.cta_state; sh.wide_cluster = o.wide_cluster == 0 ? 2 : o.wide_cluster;
    sh.wide_min = o.wide_min > 0 ? o.wide_min : 32768; sh.plain_launch = c->plainMode;
    DISPATCH(c, applyShape, c, sh);
    if (o.tune) DISPATCH(c, tuneCtx, c);
    size_t total = c->bytes + (sizeof(InstDesc) + sizeof(InstCtl) + 8) * n_instances;
    if (o.budget_bytes && total > o.budget_bytes) throw std::bad_alloc();
    CK(cudaStreamSynchronize(c->st));
  });
  if (rc == WS_ERR_NOMEM && o.budget_bytes) fail(WS_ERR_NOMEM, "ws_create: the batch needs more device memory than the budget");
  if (rc != WS_OK) { destroyCtx(c); return rc; }
  *out = c;
  return WS_OK;
}

int ws_step(ws_ctx *c, int32_t n_iter, const uint8_t *mask, ws_control *ctl) {
  if (!c || n_iter < 0) return fail(WS_ERR_ARG, "ws_step: bad arguments");
  return guarded("ws_step", [&]() {
    CK(cudaSetDevice(c->device));
    DISPATCH(c, stepImpl, c, n_iter, mask);
    c->lastMs = -1;
    if (ctl) {
      readCtl(c);
      for (size_t b = 0; b < c->inst.size(); b++) fillControl(c->ctlHost[b], c->extHost[b], ctl + b, stepStart(c));
    }
  });
}

int ws_read_control(ws_ctx *c, ws_control *ctl) {
  if (!c || !ctl) return fail(WS_ERR_ARG, "ws_read_control: bad arguments");
  return guarded("ws_read_control", [&]() {
    readCtl(c);
    for (size_t b = 0; b < c->inst.size(); b++) fillControl(c->ctlHost[b], c->extHost[b], ctl + b, stepStart(c));
  });
}

int ws_download(ws_ctx *c, int32_t b, ws_state_out *o) {
  if (!c || !o || b < 0 || b >= int(c->inst.size())) return fail(WS_ERR_ARG, "ws_download: bad instance");
  return guarded("ws_download", [&]() { DISPATCH(c, downloadImpl, c, b, o); });
}

int ws_upload_state(ws_ctx *c, int32_t b, const double *X, const double *Q, const double *u) {
  if (!c || !X || !Q || b < 0 || b >= int(c->inst.size())) return fail(WS_ERR_ARG, "ws_upload_state: bad arguments");
  return guarded("ws_upload_state", [&]() { DISPATCH(c, uploadStateImpl, c, b, X, Q, u); });
}

int ws_set_params(ws_ctx *c, int32_t b, const ws_model *md) {
  if (!c || !md || b < 0 || b >= int(c->inst.size())) return fail(WS_ERR_ARG, "ws_set_params: bad arguments");
  return guarded("ws_set_params", [&]() { DISPATCH(c, setParamsImpl, c, b, md); });
}

int ws_load_instance(ws_ctx *c, int32_t b, const ws_model *md) {
  if (!c || !md || b < 0 || b >= int(c->inst.size())) return fail(WS_ERR_ARG, "ws_load_instance: bad arguments");
  return guarded("ws_load_instance", [&]() { DISPATCH(c, loadInstanceImpl, c, b, md); });
}

int ws_internalize(ws_ctx *c, int32_t b) {
  if (!c || b < 0 || b >= int(c->inst.size())) return fail(WS_ERR_ARG, "ws_internalize: bad instance");
  return guarded("ws_internalize", [&]() { DISPATCH(c, internalizeImpl, c, b); });
}

void *ws_stream(ws_ctx *c) { return c ? c->st : nullptr; }
uint64_t ws_device_bytes(const ws_ctx *c) { return c ? c->bytes : 0; }
int ws_side_order(const ws_ctx *c) { return c && c->shortSides ? 1 : 0; }
int ws_cta_resident(const ws_ctx *c) { return c && c->residentBytes ? 1 : 0; }
int ws_get_shape(const ws_ctx *c, ws_shape *out) {
  if (!c || !out) return fail(WS_ERR_ARG, "ws_get_shape: bad arguments");
  *out = c->launch;
  return WS_OK;
}

// the tuner's view of a batch that has no context yet: host goals and descriptors only, nothing on a device
static int infoFromModels(const ws_model *const *models, int32_t n, const ws_opts *opts, TuneInfo *out, const char *who) {
  if (!models || n <= 0 || !out) return fail(WS_ERR_ARG, std::string(who) + ": need at least one model");
  ws_opts o{};
  if (opts) o = *opts;
  if (o.form < 0 || o.form > 2 || o.precision < 0 || o.precision > 2) return fail(WS_ERR_ARG, std::string(who) + ": bad options");
  return guarded(who, [&]() {
    ws_ctx tmp;
    tmp.form = o.form; tmp.prec = o.precision;
    tmp.sidesGeneral = o.side_order == WS_SIDES_GENERAL;
    tmp.g.resize(n);
    Sizes off;
    for (int b = 0; b < n; b++) {
      if (!models[b]) throw std::invalid_argument("null model");
      tmp.g[b].build(*models[b]);
      off.b = b;
      tmp.inst.push_back(describe(tmp.g[b], off));
      off.n += tmp.g[b].n; off.m += tmp.g[b].m; off.p += tmp.g[b].p; off.c += tmp.g[b].C; off.k += tmp.g[b].K; off.s += tmp.g[b].S;
    }
    tmp.shortSides = shortOrderOK(&tmp);
    *out = tuneInfo(&tmp);
  });
}

int ws_tune_key(const ws_model *const *models, int32_t n, const ws_opts *opts, const char *device, char *buf, size_t cap) {
  TuneInfo t;
  int rc = infoFromModels(models, n, opts, &t, "ws_tune_key");
  if (rc != WS_OK) return rc;
  std::string dev;
  if (device) {
    dev = device;
  } else {
    int d = 0;
    dev = (ws_device_count() > 0 && cudaGetDevice(&d) == cudaSuccess) ? deviceName(d) : "none";
  }
  const std::string k = tuneKey(dev, t);
  if (!buf || cap < k.size() + 1) return fail(WS_ERR_ARG, "ws_tune_key: buffer too small");
  std::memcpy(buf, k.c_str(), k.size() + 1);
  return WS_OK;
}

int ws_tune_candidates(const ws_model *const *models, int32_t n, const ws_opts *opts, const ws_shape *after, ws_shape *out,
                       int32_t cap) {
  TuneInfo t;
  int rc = infoFromModels(models, n, opts, &t, "ws_tune_candidates");
  if (rc != WS_OK) return rc;
  const std::vector<ws_shape> v = after ? tuneStage2(t, *after) : tuneStage1(t);
  for (int i = 0; i < int(v.size()) && i < cap && out; i++) out[i] = v[i];
  return int(v.size());
}

int ws_tune_cache_get(const char *key, ws_shape *out) {
  if (!key) return fail(WS_ERR_ARG, "ws_tune_cache_get: null key");
  return tuneLookup(key, out) ? 1 : 0;
}
int ws_tune_cache_put(const char *key, const ws_shape *shape) {
  if (!key || !shape || !*key || std::strchr(key, ' ') || std::strchr(key, '\n'))
    return fail(WS_ERR_ARG, "ws_tune_cache_put: a key is one word");
  tuneStore(key, *shape);
  return WS_OK;
}
int ws_tune_cache_clear(void) {
  tuneClear();
  return WS_OK;
}

int ws_wide_instances(const ws_ctx *c, int32_t *cluster) {
  if (cluster) *cluster = c ? c->wideCl : 0;
  return c ? c->nWide : 0;
}
int ws_last_step_stats(const ws_ctx *c_, double *ms, int64_t *launches) {
  if (!c_) return fail(WS_ERR_ARG, "ws_last_step_stats: null context");
  ws_ctx *c = const_cast<ws_ctx *>(c_);
  if (c->lastMs < 0) {
    float t = 0;
    if (cudaEventSynchronize(c->ev1) != cudaSuccess || cudaEventElapsedTime(&t, c->ev0, c->ev1) != cudaSuccess)
      return fail(WS_ERR_CUDA, "ws_last_step_stats: event timing failed");
    c->lastMs = t;
  }
  if (ms) *ms = c->lastMs;
  if (launches) *launches = c->lastLaunches;
  return WS_OK;
}
int ws_destroy(ws_ctx *c) {
  if (!c) return WS_OK;
  cudaSetDevice(c->device);
  destroyCtx(c);
  return WS_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------ caller-provided memory
// Runs one instance whose whole device footprint (arena, descriptor, control block) lives in memory the caller hands
// over (`base`, `cap` bytes): set-up, `n_iter` iterations of the batched kernel, download.  Used by the allocation-free
// entry point (capi_noalloc.cu); nothing here allocates device memory.
namespace wsb {

// the end of the arena inside caller-provided memory: the same 4096 spare bytes after the last array as ws_create's
// arena has, then 256-byte alignment for the descriptor and control block that follow
static size_t arenaEnd(size_t carved) { return (carved + 4096 + 255) & ~size_t(255); }

size_t instanceFootprint(int prec, const HostGoals &g) {
  Sizes z;
  z.n = g.n; z.m = g.m; z.p = g.p; z.c = g.C; z.k = g.K; z.s = g.S; z.b = 1;
  Carver cv{nullptr};
  switch (prec) {
    case WS_PREC_F64: { Dev<PREC_F64> d{}; layout<PREC_F64>(d, cv, z); break; }
    case WS_PREC_MIXED: { Dev<PREC_MIXED> d{}; layout<PREC_MIXED>(d, cv, z); break; }
    default: { Dev<PREC_F32> d{}; layout<PREC_F32>(d, cv, z); break; }
  }
  const size_t tail = ((sizeof(InstDesc) + 255) & ~size_t(255)) + ((sizeof(InstCtl) + 255) & ~size_t(255));
  return arenaEnd(cv.off) + tail;
}

template <int P>
static void runInPlaceImpl(ws_ctx *c, char *base, int nIter, int threads, ws_state_out *out, ws_control *ctl) {
  Carver cv{base};
  layout<P>(devOf<P>(c), cv, c->z);
  c->dExt = devOf<P>(c).ext;
  const size_t off = arenaEnd(cv.off);
  c->dInst = reinterpret_cast<InstDesc *>(base + off);
  c->dCtl = reinterpret_cast<InstCtl *>(base + off + ((sizeof(InstDesc) + 255) & ~size_t(255)));
  CK(cudaMemsetAsync(base, 0, off, c->st));
  CK(cudaMemcpyAsync(c->dInst, c->inst.data(), sizeof(InstDesc), cudaMemcpyHostToDevice, c->st));
  InstCtl s;
  std::memset(&s, 0, sizeof(s));
  s.status = WS_RUNNING; s.residual = INFINITY;
  CK(cudaMemcpyAsync(c->dCtl, &s, sizeof(InstCtl), cudaMemcpyHostToDevice, c->st));
  uploadAll<P>(c);
  if (nIter > 0)
    CK(launchBatched<P>(devOf<P>(c), c->dInst, c->dCtl, nullptr, 1, nIter, nullptr, threads, 1, c->shortSides, anyExt(c), c->st));
  CK(cudaStreamSynchronize(c->st));
  if (out) downloadImpl<P>(c, 0, out);
  if (ctl) { readCtl(c); fillControl(c->ctlHost[0], c->extHost[0], ctl, stepStart(c)); }
}

int runInPlace(int prec, const HostGoals &g, char *base, int nIter, int threads, cudaStream_t st, ws_state_out *out,
               ws_control *ctl, std::string &err) {
  ws_ctx tmp;                       // host-side bookkeeping only: its device pointers point into `base`
  tmp.prec = prec; tmp.form = WS_FORM_CTA; tmp.threads = threads; tmp.st = st;
  tmp.g.push_back(g);
  Sizes off;
  tmp.inst.push_back(describe(tmp.g[0], off));
  tmp.z.n = g.n; tmp.z.m = g.m; tmp.z.p = g.p; tmp.z.c = g.C; tmp.z.k = g.K; tmp.z.s = g.S; tmp.z.b = 1;
  tmp.shortSides = shortOrderOK(&tmp);
  try {
    switch (prec) {
      case WS_PREC_F64: runInPlaceImpl<PREC_F64>(&tmp, base, nIter, threads, out, ctl); break;
      case WS_PREC_MIXED: runInPlaceImpl<PREC_MIXED>(&tmp, base, nIter, threads, out, ctl); break;
      default: runInPlaceImpl<PREC_F32>(&tmp, base, nIter, threads, out, ctl); break;
    }
  } catch (const std::exception &e) {
    dropPuts();
    err = e.what();
    return WS_ERR_CUDA;
  }
  return WS_OK;
}

}  // namespace wsb
