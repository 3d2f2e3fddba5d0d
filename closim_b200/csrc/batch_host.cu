// Host side of the batched solver (cs_batch_*): packs many independent
// sheets into one work list, steps them with one persistent launch per step
// (captured into a CUDA graph for multi-step calls) and picks the launch's
// block size by timing the candidates on the batch itself.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/closim_batch.h"
#include "batch.cuh"
#include "setup.hpp"

namespace cs {
namespace {

struct BErr : std::runtime_error {
  int code;
  BErr(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};
#define BK(call)                                                               \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) throw cs::BErr(CS_E_CUDA, cudaGetErrorString(e_));  \
  } while (0)

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t k) {
    free();
    n = k;
    if (k) BK(cudaMalloc(&p, k * sizeof(T)));
  }
  void up(const T* h, size_t k, cudaStream_t s) {
    alloc(std::max<size_t>(k, 1));
    if (k) BK(cudaMemcpyAsync(p, h, k * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~Buf() { free(); }
};

}  // namespace

struct Batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int S = 0, N = 0, M = 0, HG = 0;
  Buf<int> vStart, tStart, hStart, order;
  Buf<uint32_t> idx, memOff, memRec, hinOff, hinRec;
  Buf<float4> inv;
  Buf<float> area, mass;
  Buf<int4> hinge;
  Buf<double> hmeta, pinPos, mat;
  Buf<uint8_t> pinned, act, lagOk;
  Buf<double> x, v, x0, yHat, g, dx, xt, diag, elem, helem, lagLam, out;
  Buf<float> r, z, p, Ap, xs, tris, dinv;
  Buf<unsigned int> work;
  BatchDev d{};
  cs_stepper_options opts{10, 60, 10, CS_PRECOND_JACOBI, 1e-5};
  cs_contact_params cp{1e-3, 50.0, 1e-4, 0.3, 1e-4};
  int floorOn = 0;
  double floorY = 0;
  double gravity[3] = {0, -9.81, 0};
  std::vector<double> matRows;  // S x BM_N, host copy
  int threads = 512;
  int ctas = 0;
  bool ready = false;
  cudaGraphExec_t graph = nullptr;
  int graphSteps = 0;
  double graphH = 0;
  std::string err;
  std::vector<double> hout;

  ~Batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }

  void drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graphSteps = 0;
  }

  void initialize(int sheets, const cs_mesh* meshes, const cs_material* mats, const double* hx, const double* hv,
                  const int32_t* pinCounts, const int32_t* pinIds, const double* pinP, const double* grav) {
    if (sheets <= 0 || !meshes || !mats || !hx) throw BErr(CS_E_ARG, "empty batch");
    drop_graph();
    ready = false;
    S = sheets;
    std::vector<int> vs(S + 1, 0), ts(S + 1, 0), hs(S + 1, 0);
    for (int s = 0; s < S; s++) {
      const cs_mesh& m = meshes[s];
      if (m.n <= 0 || m.m <= 0 || m.hg < 0 || !m.indices || !m.inv_dm || !m.area || !m.mass ||
          (m.hg > 0 && (!m.hinge || !m.hinge_meta)))
        throw BErr(CS_E_ARG, "bad mesh for sheet " + std::to_string(s));
      vs[s + 1] = vs[s] + m.n;
      ts[s + 1] = ts[s] + m.m;
      hs[s + 1] = hs[s] + m.hg;
    }
    N = vs[S]; M = ts[S]; HG = hs[S];
    if ((long)M * 4 >= (1l << 32) || (long)HG * 4 >= (1l << 32)) throw BErr(CS_E_CAPACITY, "batch too large");
    // packed union mesh (global vertex ids) and its incidence
    HostMesh u;
    u.n = N; u.m = M; u.hg = HG;
    u.idx.resize(3 * (size_t)M);
    u.hinge.resize(4 * (size_t)HG);
    std::vector<float> inv4(4 * (size_t)M), ar(M), ms(N);
    std::vector<double> hm(3 * (size_t)HG);
    std::vector<uint8_t> pin(N, 0);
    std::vector<double> pp(3 * (size_t)N, 0.0);
    matRows.assign((size_t)S * BM_N, 0.0);
    int pinCursor = 0;
    for (int s = 0; s < S; s++) {
      const cs_mesh& m = meshes[s];
      for (int q = 0; q < 3 * m.m; q++) {
        if ((int)m.indices[q] >= m.n) throw BErr(CS_E_ARG, "triangle index out of range");
        u.idx[3 * (size_t)ts[s] + q] = m.indices[q] + (uint32_t)vs[s];
      }
      std::memcpy(inv4.data() + 4 * (size_t)ts[s], m.inv_dm, 16 * (size_t)m.m);
      std::memcpy(ar.data() + ts[s], m.area, 4 * (size_t)m.m);
      std::memcpy(ms.data() + vs[s], m.mass, 4 * (size_t)m.n);
      for (int q = 0; q < 4 * m.hg; q++) {
        if (m.hinge[q] < 0 || m.hinge[q] >= m.n) throw BErr(CS_E_ARG, "hinge index out of range");
        u.hinge[4 * (size_t)hs[s] + q] = m.hinge[q] + vs[s];
      }
      if (m.hg) std::memcpy(hm.data() + 3 * (size_t)hs[s], m.hinge_meta, 24 * (size_t)m.hg);
      const cs_material& mt = mats[s];
      double* row = matRows.data() + (size_t)s * BM_N;
      row[BM_C00] = mt.stretch_warp; row[BM_C11] = mt.stretch_weft; row[BM_C01] = mt.stretch_coupling;
      row[BM_G] = mt.shear; row[BM_THICK] = mt.thickness; row[BM_KB] = 0.5 * (mt.bend_warp + mt.bend_weft);
      row[BM_DAMP] = 1 - std::min(std::max(mt.damping, 0.0), 0.1);
      row[BM_BETA] = std::max(std::max(mt.stretch_warp, mt.stretch_weft), mt.shear) * mt.thickness * 0.1 + 1e-6;
      const int k = pinCounts ? pinCounts[s] : 0;
      for (int q = 0; q < k; q++) {
        const int id = pinIds[pinCursor + q];
        if (id < 0 || id >= m.n) throw BErr(CS_E_ARG, "pin id out of range");
        pin[vs[s] + id] = 1;
        for (int c = 0; c < 3; c++) pp[3 * (size_t)(vs[s] + id) + c] = pinP[3 * (size_t)(pinCursor + q) + c];
      }
      pinCursor += k;
    }
    build_topology(u);
    if (!stream) {
      BK(cudaSetDevice(device));
      BK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    }
    std::vector<int> ord(S);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return ts[a + 1] - ts[a] > ts[b + 1] - ts[b]; });
    cudaStream_t st = stream;
    vStart.up(vs.data(), vs.size(), st); tStart.up(ts.data(), ts.size(), st); hStart.up(hs.data(), hs.size(), st);
    order.up(ord.data(), ord.size(), st);
    idx.up(u.idx.data(), u.idx.size(), st);
    inv.up(reinterpret_cast<const float4*>(inv4.data()), M, st);
    area.up(ar.data(), M, st);
    mass.up(ms.data(), N, st);
    hinge.up(reinterpret_cast<const int4*>(u.hinge.data()), HG, st);
    hmeta.up(hm.data(), hm.size(), st);
    memOff.up(u.memOff.data(), u.memOff.size(), st);
    memRec.up(u.memRec.data(), u.memRec.size(), st);
    hinOff.up(u.hinOff.data(), u.hinOff.size(), st);
    hinRec.up(u.hinRec.data(), u.hinRec.size(), st);
    pinned.up(pin.data(), N, st);
    pinPos.up(pp.data(), pp.size(), st);
    mat.up(matRows.data(), matRows.size(), st);
    const size_t n3 = 3 * (size_t)N;
    x.up(hx, n3, st);
    v.alloc(n3);
    if (hv) BK(cudaMemcpyAsync(v.p, hv, n3 * 8, cudaMemcpyHostToDevice, st));
    else BK(cudaMemsetAsync(v.p, 0, n3 * 8, st));
    for (Buf<double>* b : {&x0, &yHat, &g, &dx, &xt, &diag}) b->alloc(n3);
    elem.alloc(9 * (size_t)M);
    helem.alloc(12 * (size_t)std::max(HG, 1));
    for (Buf<float>* b : {&r, &z, &p, &Ap, &xs, &dinv}) b->alloc(n3);
    tris.alloc(16 * (size_t)M);
    act.alloc(N);
    BK(cudaMemsetAsync(act.p, 0, N, st));
    lagOk.alloc(N);
    BK(cudaMemsetAsync(lagOk.p, 0, N, st));
    lagLam.alloc(N);
    out.alloc((size_t)S * BO_N);
    BK(cudaMemsetAsync(out.p, 0, (size_t)S * BO_N * 8, st));
    work.alloc(1);
    if (grav) for (int k = 0; k < 3; k++) gravity[k] = grav[k];
    BK(cudaStreamSynchronize(st));
    ctas = batch_max_ctas(threads);
    ready = true;
  }

  void bind(double h) {
    d = BatchDev{};
    d.S = S; d.vStart = vStart.p; d.tStart = tStart.p; d.hStart = hStart.p; d.order = order.p;
    d.idx = idx.p; d.inv = inv.p; d.area = area.p; d.mass = mass.p; d.hinge = hinge.p; d.hmeta = hmeta.p;
    d.memOff = memOff.p; d.memRec = memRec.p; d.hinOff = hinOff.p; d.hinRec = hinRec.p;
    d.pinned = pinned.p; d.pinPos = pinPos.p; d.mat = mat.p;
    d.x = x.p; d.v = v.p; d.x0 = x0.p; d.yHat = yHat.p; d.g = g.p; d.dx = dx.p; d.xt = xt.p; d.diag = diag.p;
    d.elem = elem.p; d.helem = helem.p;
    d.r = r.p; d.z = z.p; d.p = p.p; d.Ap = Ap.p; d.xs = xs.p; d.tris = tris.p; d.dinv = dinv.p;
    d.act = act.p; d.lagLam = lagLam.p; d.lagOk = lagOk.p;
    d.hasFloor = floorOn; d.floorY = floorY;
    d.dHat = cp.dhat; d.kappa = cp.kappa; d.dMin = cp.dmin; d.mu = cp.mu; d.eps = cp.eps;
    d.h = h; d.invH2 = 1 / (h * h);
    for (int k = 0; k < 3; k++) d.gravity[k] = gravity[k];
    d.newtonIters = opts.newton_iters; d.pcgMaxIters = opts.pcg_max_iters; d.lsIters = opts.ls_iters;
    d.gradTol = opts.grad_tol;
    d.out = out.p; d.work = work.p;
  }

  // One step = reset of the work list + one persistent launch.
  void enqueue_step(double h) {
    bind(h);
    BK((cudaError_t)batch_launch_step(d, threads, ctas, stream));
  }

  void step(double h, int steps) {
    if (!ready) throw BErr(CS_E_UNINIT, "batch not initialized");
    if (steps <= 0) throw BErr(CS_E_ARG, "steps must be positive");
    if (steps == 1) {
      enqueue_step(h);
    } else {
      // the step sequence is captured once into a graph and replayed
      if (!graph || graphSteps != steps || graphH != h) {
        drop_graph();
        cudaGraph_t gr = nullptr;
        BK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
          for (int k = 0; k < steps; k++) enqueue_step(h);
        } catch (...) {
          cudaStreamEndCapture(stream, &gr);
          if (gr) cudaGraphDestroy(gr);
          throw;
        }
        BK(cudaStreamEndCapture(stream, &gr));
        const cudaError_t e = cudaGraphInstantiate(&graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) { graph = nullptr; throw BErr(CS_E_CUDA, cudaGetErrorString(e)); }
        graphSteps = steps;
        graphH = h;
      }
      BK(cudaGraphLaunch(graph, stream));
    }
    BK(cudaStreamSynchronize(stream));
  }

  // Times one step for each block size on a copy of the state, keeps the fastest.
  int autotune(double h) {
    if (!ready) throw BErr(CS_E_UNINIT, "batch not initialized");
    const size_t n3 = 3 * (size_t)N;
    Buf<double> sx, sv, sl;
    Buf<uint8_t> so;
    sx.alloc(n3); sv.alloc(n3); sl.alloc(N); so.alloc(N);
    BK(cudaMemcpyAsync(sx.p, x.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    BK(cudaMemcpyAsync(sv.p, v.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    BK(cudaMemcpyAsync(sl.p, lagLam.p, (size_t)N * 8, cudaMemcpyDeviceToDevice, stream));
    BK(cudaMemcpyAsync(so.p, lagOk.p, (size_t)N, cudaMemcpyDeviceToDevice, stream));
    cudaEvent_t e0, e1;
    BK(cudaEventCreate(&e0));
    BK(cudaEventCreate(&e1));
    // Candidates: block size (vertices per thread of a sheet) x number of
    // resident blocks (sheets in flight per SM). Fewer blocks keep fewer sheets
    // in flight, so their working sets can stay in L2. Every candidate compiles
    // without register spills (1024 threads would cap a thread at 64 registers).
    const int cands[3] = {128, 256, 512};
    const int fracs[3] = {1, 2, 3};
    float best = 1e30f;
    int bestT = threads, bestC = ctas;
    drop_graph();
    for (int ci = 0; ci < 9; ci++) {
      const int T = cands[ci / 3];
      threads = T;
      ctas = std::max(1, batch_max_ctas(T) / fracs[ci % 3]);
      BK(cudaMemcpyAsync(x.p, sx.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
      BK(cudaMemcpyAsync(v.p, sv.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
      BK(cudaMemcpyAsync(lagLam.p, sl.p, (size_t)N * 8, cudaMemcpyDeviceToDevice, stream));
      BK(cudaMemcpyAsync(lagOk.p, so.p, (size_t)N, cudaMemcpyDeviceToDevice, stream));
      BK(cudaEventRecord(e0, stream));
      enqueue_step(h);
      BK(cudaEventRecord(e1, stream));
      BK(cudaEventSynchronize(e1));
      float ms = 0;
      BK(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) { best = ms; bestT = T; bestC = ctas; }
    }
    BK(cudaMemcpyAsync(x.p, sx.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    BK(cudaMemcpyAsync(v.p, sv.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    BK(cudaMemcpyAsync(lagLam.p, sl.p, (size_t)N * 8, cudaMemcpyDeviceToDevice, stream));
    BK(cudaMemcpyAsync(lagOk.p, so.p, (size_t)N, cudaMemcpyDeviceToDevice, stream));
    BK(cudaStreamSynchronize(stream));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    threads = bestT;
    ctas = bestC;
    return bestT;
  }
};

}  // namespace cs

namespace {
template <class F>
int bguard(cs::Batch* b, F&& f) {
  if (!b) return CS_E_ARG;
  try {
    f();
    b->err.clear();
    return CS_OK;
  } catch (const cs::BErr& e) {
    b->err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    b->err = "host allocation failed";
    return CS_E_CAPACITY;
  } catch (const std::exception& e) {
    b->err = e.what();
    return CS_E_CUDA;
  }
}
cs::Batch* B(cs_batch* h) { return reinterpret_cast<cs::Batch*>(h); }
}  // namespace

extern "C" {

cs_batch* cs_batch_create(int32_t device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return nullptr;
  }
  cs::Batch* b = new (std::nothrow) cs::Batch();
  if (b) b->device = device;
  return reinterpret_cast<cs_batch*>(b);
}

void cs_batch_destroy(cs_batch* h) { delete B(h); }

const char* cs_batch_last_error(cs_batch* h) { return h ? B(h)->err.c_str() : "null batch handle"; }

int cs_batch_initialize(cs_batch* h, int32_t sheets, const cs_mesh* meshes, const cs_material* mats, const double* x,
                        const double* v, const int32_t* pin_counts, const int32_t* pin_ids, const double* pin_pos,
                        const double* gravity) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    cudaSetDevice(b->device);
    b->initialize(sheets, meshes, mats, x, v, pin_counts, pin_ids, pin_pos, gravity);
  });
}

int cs_batch_set_contact(cs_batch* h, const cs_contact_params* p, int32_t floor_on, double floor_y) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (!p || !(p->dhat > 0) || !(p->dmin >= 0) || !(p->kappa >= 0) || !(p->eps > 0) || !(p->mu >= 0))
      throw cs::BErr(CS_E_ARG, "bad contact parameters");
    b->cp = *p;
    b->floorOn = floor_on != 0;
    b->floorY = floor_y;
    b->drop_graph();
  });
}

int cs_batch_set_stepper_options(cs_batch* h, const cs_stepper_options* o) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (!o || o->newton_iters <= 0 || o->pcg_max_iters <= 0 || o->ls_iters <= 0 || !(o->grad_tol >= 0))
      throw cs::BErr(CS_E_ARG, "bad stepper options");
    if (o->precond != CS_PRECOND_JACOBI) throw cs::BErr(CS_E_ARG, "the batched solver uses the Jacobi preconditioner");
    b->opts = *o;
    b->drop_graph();
  });
}

int cs_batch_step(cs_batch* h, double dt, int32_t steps) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    cudaSetDevice(b->device);
    if (!(dt > 0)) throw cs::BErr(CS_E_ARG, "dt must be positive");
    b->step(dt, steps);
  });
}

int cs_batch_get_positions(cs_batch* h, double* out) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (!b->ready) throw cs::BErr(CS_E_UNINIT, "batch not initialized");
    BK(cudaMemcpy(out, b->x.p, 3 * (size_t)b->N * 8, cudaMemcpyDeviceToHost));
  });
}

int cs_batch_get_velocities(cs_batch* h, double* out) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (!b->ready) throw cs::BErr(CS_E_UNINIT, "batch not initialized");
    BK(cudaMemcpy(out, b->v.p, 3 * (size_t)b->N * 8, cudaMemcpyDeviceToHost));
  });
}

int cs_batch_stats(cs_batch* h, double* out) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (!b->ready) throw cs::BErr(CS_E_UNINIT, "batch not initialized");
    BK(cudaMemcpy(out, b->out.p, (size_t)b->S * cs::BO_N * 8, cudaMemcpyDeviceToHost));
  });
}

int cs_batch_autotune(cs_batch* h, double dt, int32_t* threads) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    cudaSetDevice(b->device);
    const int t = b->autotune(dt);
    if (threads) *threads = t;
  });
}

int cs_batch_set_threads(cs_batch* h, int32_t threads) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (threads != 128 && threads != 256 && threads != 512) throw cs::BErr(CS_E_ARG, "threads: 128, 256 or 512");
    b->threads = threads;
    b->ctas = b->ready ? cs::batch_max_ctas(threads) : 0;
    b->drop_graph();
  });
}

int cs_batch_launch_shape(cs_batch* h, int32_t* threads, int32_t* blocks) {
  cs::Batch* b = B(h);
  return bguard(b, [&] {
    if (threads) *threads = b->threads;
    if (blocks) *blocks = b->ctas;
  });
}

void* cs_batch_stream(cs_batch* h) { return h ? (void*)B(h)->stream : nullptr; }

}  // extern "C"
