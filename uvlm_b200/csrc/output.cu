// output.cu -- per-step state output of the time-stepper in the reference's
// protobuf messages (proto/uvlm.proto): AllVortexSheets
// (SimpleSimulator::OutputSheet, src/simulator/simple_simulator.cpp:324-332,
// proto_adaptor::ToVortexSheet src/proto_adaptor.h:116-137) and Snapshot2
// (OutputPanels :317-322, output::SheetToSnapshot src/output.cpp:11-32).
//
// The state is snapshotted on the compute stream into a device staging slot
// (a few device-to-device copies), copied to pinned host memory on a side
// stream, and serialised and written by a writer thread, so the time-stepper
// does not wait for the file system.  Two slots: a step waits only when both
// previous snapshots are still being written.
//
// Framing: every record is its byte length (uint64, little endian) followed by
// the serialised message.  (The reference frames records with its recordio
// submodule, whose source is not part of the reference tree.)
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

#include "output.cuh"

namespace uvlm {
namespace {

// ------------------------------------------------------- wire encoding
void put_varint(std::string& o, unsigned long long v) {
  while (v >= 0x80) {
    o.push_back((char)(v | 0x80));
    v >>= 7;
  }
  o.push_back((char)v);
}
void put_tag(std::string& o, int field, int wire) { put_varint(o, ((unsigned long long)field << 3) | wire); }
void put_double(std::string& o, int field, double d) {
  put_tag(o, field, 1);
  unsigned char b[8];
  std::memcpy(b, &d, 8);  // IEEE-754, little-endian host
  o.append(reinterpret_cast<const char*>(b), 8);
}
void put_uint(std::string& o, int field, unsigned long long v) {
  put_tag(o, field, 0);
  put_varint(o, v);
}
void put_bytes(std::string& o, int field, const std::string& body) {
  put_tag(o, field, 2);
  put_varint(o, body.size());
  o += body;
}
// proto::Point {x = 1, y = 2, z = 3}
void put_point(std::string& o, int field, const double* p) {
  std::string b;
  put_double(b, 1, p[0]);
  put_double(b, 2, p[1]);
  put_double(b, 3, p[2]);
  put_bytes(o, field, b);
}
// proto::VortexRing {gamma = 1, nodes = 2 (repeated)} (VortexRingToProto,
// src/proto_adaptor.h:26-37; nodes0 is empty for sheet rings)
void put_ring(std::string& o, int field, double gamma, const double* const nodes[4]) {
  std::string b;
  put_double(b, 1, gamma);
  for (int q = 0; q < 4; ++q) put_point(b, 2, nodes[q]);
  put_bytes(o, field, b);
}

// Ring (n, i, j) of a sheet: p(i,j), p(i,j+1), p(i+1,j+1), p(i+1,j).
struct SheetRef {
  int num, rows, cols;   // rings per sheet: rows x cols
  const double* pos;     // [num][rows+1][cols+1][3]
  const double* gamma;   // [num][rows][cols]
  const double* p(int n, int i, int j) const { return pos + 3 * (((long long)n * (rows + 1) + i) * (cols + 1) + j); }
  double g(int n, int i, int j) const { return gamma[((long long)n * rows + i) * cols + j]; }
};

// proto::VortexSheet {num = 2, rows = 3, cols = 4, vortices = 5} (ToVortexSheet)
std::string vortex_sheet(const SheetRef& s) {
  std::string o;
  put_uint(o, 2, (unsigned)s.num);
  put_uint(o, 3, (unsigned)s.rows);
  put_uint(o, 4, (unsigned)s.cols);
  for (int n = 0; n < s.num; ++n)
    for (int i = 0; i < s.rows; ++i)
      for (int j = 0; j < s.cols; ++j) {
        const double* nodes[4] = {s.p(n, i, j), s.p(n, i, j + 1), s.p(n, i + 1, j + 1), s.p(n, i + 1, j)};
        put_ring(o, 5, s.g(n, i, j), nodes);
      }
  return o;
}

// Snapshot2.vortices (field 3) of one sheet set, nodes in SheetToSnapshot's
// order p(i+1,j), p(i+1,j+1), p(i,j+1), p(i,j).
void snapshot_rings(std::string& o, const SheetRef& s) {
  for (int n = 0; n < s.num; ++n)
    for (int i = 0; i < s.rows; ++i)
      for (int j = 0; j < s.cols; ++j) {
        const double* nodes[4] = {s.p(n, i + 1, j), s.p(n, i + 1, j + 1), s.p(n, i, j + 1), s.p(n, i, j)};
        put_ring(o, 3, s.g(n, i, j), nodes);
      }
}

std::string encode(int kind, const SheetRef& wing, const SheetRef& wake, double t) {
  std::string o;
  if (kind == UVLM_OUTPUT_SHEETS) {  // AllVortexSheets {t = 1, wing = 2, wake = 3}
    put_double(o, 1, t);
    put_bytes(o, 2, vortex_sheet(wing));
    put_bytes(o, 3, vortex_sheet(wake));
  } else {  // Snapshot2: vortices only (OutputPanels sets nothing else)
    snapshot_rings(o, wing);
    snapshot_rings(o, wake);
  }
  return o;
}

// proto::VortexRing of the legacy pool with its reference nodes
// (VortexRingToProto, src/proto_adaptor.h:29-40): gamma, nodes, nodes0.
void put_pool_ring(std::string& o, int field, double gamma, const double* nodes, const double* nodes0) {
  std::string b;
  put_double(b, 1, gamma);
  for (int q = 0; q < 4; ++q) put_point(b, 2, nodes + 3 * q);
  if (nodes0)
    for (int q = 0; q < 4; ++q) put_point(b, 3, nodes0 + 3 * q);
  put_bytes(o, field, b);
}

bool write_record(FILE* f, const std::string& msg) {
  unsigned char len[8];
  unsigned long long n = msg.size();
  for (int b = 0; b < 8; ++b) len[b] = (unsigned char)(n >> (8 * b));
  return fwrite(len, 1, 8, f) == 8 && fwrite(msg.data(), 1, msg.size(), f) == msg.size();
}

}  // namespace

Error output_encode_to_file(const char* path, int append, int kind, int num, int rows, int cols, int wake_rows,
                            const double* wing_pos, const double* wing_gamma, const double* wake_pos,
                            const double* wake_gamma, double t) {
  FILE* f = fopen(path, append ? "ab" : "wb");
  if (!f) return fail(kErrInvalid, std::string("cannot open ") + path);
  const SheetRef wing{num, rows, cols, wing_pos, wing_gamma};
  const SheetRef wake{num, wake_rows, cols, wake_pos, wake_gamma};
  const bool okw = write_record(f, encode(kind, wing, wake, t));
  const bool okc = fclose(f) == 0;
  return okw && okc ? ok() : fail(kErrInvalid, std::string("write failed: ") + path);
}

Error output_write_legacy_snapshot2(const char* path, double t, const LegacySnapshot& s) {
  std::string o;
  put_double(o, 1, t);
  for (long long c = 0; c < s.n_containers; ++c) {  // ContainerShape {rows 1, cols 2, id 3, chord 5, span 6}
    std::string b;
    put_uint(b, 1, (unsigned)s.rows[c]);
    put_uint(b, 2, (unsigned)s.cols[c]);
    put_uint(b, 3, (unsigned)c);
    put_double(b, 5, s.chord[c]);
    put_double(b, 6, s.span[c]);
    put_bytes(o, 2, b);
  }
  for (long long r = 0; r < s.n_rings; ++r)
    put_pool_ring(o, 3, s.gamma[r], s.rings + 12 * r, s.rings0 ? s.rings0 + 12 * r : nullptr);
  for (long long m = 0; m < s.n_mv; ++m) {  // MorphingVelocity {center 1, nodes 2, freestream 3}
    std::string b;
    put_point(b, 1, s.mv_center + 3 * m);
    for (int q = 0; q < 4; ++q) put_point(b, 2, s.mv_nodes + 12 * m + 3 * q);
    put_point(b, 3, s.mv_freestream + 3 * m);
    put_bytes(o, 4, b);
  }
  FILE* f = fopen(path, "wb");
  if (!f) return fail(kErrInvalid, std::string("Unable to open ") + path);
  const bool okw = fwrite(o.data(), 1, o.size(), f) == o.size();
  const bool okc = fclose(f) == 0;
  return okw && okc ? ok() : fail(kErrInvalid, std::string("write failed: ") + path);
}

// ------------------------------------------------------ the writer
struct OutputWriter {
  struct Meta {
    int num = 0, R = 0, C = 0, wake_nodes = 0;
    double t = 0;
  };
  struct Slot {
    double* d = nullptr;
    double* h = nullptr;
    cudaEvent_t ready = nullptr, copied = nullptr;
    bool busy = false;
    Meta meta;
  };
  FILE* files[2] = {nullptr, nullptr};  // sheets, snapshot2
  int device = 0;
  cudaStream_t os = nullptr;
  Slot slot[2];
  size_t cap = 0;  // doubles per slot
  int next = 0;
  std::thread th;
  std::mutex m;
  std::condition_variable cv;
  std::deque<int> q;
  bool stop = false;
  std::string err;

  void run() {
    cudaSetDevice(device);
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return stop || !q.empty(); });
        if (q.empty()) return;
        k = q.front();
      }
      Slot& s = slot[k];
      std::string e;
      if (cudaEventSynchronize(s.copied) != cudaSuccess) e = "output copy failed";
      if (e.empty()) {
        const Meta& M = s.meta;
        const long long nn = (long long)M.num * (M.R + 1) * (M.C + 1) * 3;
        const long long N = (long long)M.num * M.R * M.C;
        const int wr = M.wake_nodes > 0 ? M.wake_nodes - 1 : 0;
        const double* pos = s.h;
        const double* gam = pos + nn;
        const double* wpos = gam + N;
        const double* wgam = wpos + (long long)M.num * M.wake_nodes * (M.C + 1) * 3;
        const SheetRef wing{M.num, M.R, M.C, pos, gam};
        // a wake without node rows (never after the first shed) is written as 0 rows
        const SheetRef wake{M.num, wr, M.C, wpos, wgam};
        for (int kind = 0; kind < 2 && e.empty(); ++kind)
          if (files[kind] && !write_record(files[kind], encode(kind, wing, wake, M.t))) e = "output write failed";
      }
      std::lock_guard<std::mutex> lk(m);
      q.pop_front();
      s.busy = false;
      if (!e.empty() && err.empty()) err = e;
      cv.notify_all();
    }
  }
};

Error output_open(OutputWriter** out, const char* sheet_path, const char* result_path, int device) {
  *out = nullptr;
  auto* w = new OutputWriter;
  w->device = device;
  const char* paths[2] = {sheet_path, result_path};
  for (int k = 0; k < 2; ++k)
    if (paths[k] && *paths[k]) {
      w->files[k] = fopen(paths[k], "wb");
      if (!w->files[k]) {
        for (FILE* f : w->files)
          if (f) fclose(f);
        delete w;
        return fail(kErrInvalid, std::string("cannot open ") + paths[k]);
      }
    }
  if (cudaStreamCreateWithFlags(&w->os, cudaStreamNonBlocking) != cudaSuccess) {
    for (FILE* f : w->files)
      if (f) fclose(f);
    delete w;
    return fail(kErrCuda, "output stream");
  }
  w->th = std::thread([w] { w->run(); });
  *out = w;
  return ok();
}

Error output_enqueue(OutputWriter* w, const OutputState& s, double t, cudaStream_t st) {
  const long long nn = (long long)s.num * (s.R + 1) * (s.C + 1) * 3;
  const long long N = (long long)s.num * s.R * s.C;
  const int wr = s.wake_nodes > 0 ? s.wake_nodes - 1 : 0;
  const long long wn = (long long)s.wake_nodes * (s.C + 1) * 3, wg = (long long)wr * s.C;
  const size_t need = (size_t)(nn + N + s.num * (wn + wg));
  std::unique_lock<std::mutex> lk(w->m);
  w->cv.wait(lk, [&] { return !w->slot[w->next].busy || !w->err.empty(); });
  if (!w->err.empty()) return fail(kErrInvalid, w->err);
  auto& S = w->slot[w->next];
  S.busy = true;
  lk.unlock();
  auto release = [&](Error e) {
    std::lock_guard<std::mutex> g(w->m);
    S.busy = false;
    return e;
  };
  if (need > w->cap) {  // grow both slots (the wake grows with the run)
    cudaStreamSynchronize(w->os);
    const size_t cap = need + need / 4 + 4096;
    for (auto& sl : w->slot) {
      if (&sl != &S) {
        std::unique_lock<std::mutex> l2(w->m);
        w->cv.wait(l2, [&] { return !sl.busy; });
      }
      cudaFree(sl.d);
      cudaFreeHost(sl.h);
      sl.d = nullptr;
      sl.h = nullptr;
      if (cudaMalloc(&sl.d, sizeof(double) * cap) != cudaSuccess ||
          cudaMallocHost(&sl.h, sizeof(double) * cap) != cudaSuccess)
        return release(fail(kErrCuda, "output staging allocation failed"));
      if (!sl.ready && (cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming) != cudaSuccess ||
                        cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming) != cudaSuccess))
        return release(fail(kErrCuda, "output events"));
    }
    w->cap = cap;
  }
  double* d = S.d;
  auto dd = [&](double* dst, const double* src, long long cnt) -> bool {
    return cnt == 0 || cudaMemcpyAsync(dst, src, sizeof(double) * cnt, cudaMemcpyDeviceToDevice, st) == cudaSuccess;
  };
  bool okc = dd(d, s.pos, nn) && dd(d + nn, s.gamma, N);
  double* dw = d + nn + N;
  double* dg = dw + s.num * wn;
  for (int n = 0; n < s.num && okc; ++n) {
    okc = dd(dw + n * wn, s.wpos + ((long long)n * s.PR + s.wake_start) * (s.C + 1) * 3, wn) &&
          dd(dg + n * wg, s.wgamma + ((long long)n * s.PR + s.wake_start) * s.C, wg);
  }
  okc = okc && cudaEventRecord(S.ready, st) == cudaSuccess && cudaStreamWaitEvent(w->os, S.ready, 0) == cudaSuccess &&
        cudaMemcpyAsync(S.h, d, sizeof(double) * need, cudaMemcpyDeviceToHost, w->os) == cudaSuccess &&
        cudaEventRecord(S.copied, w->os) == cudaSuccess;
  if (!okc) return release(fail(kErrCuda, "output snapshot copies failed"));
  S.meta = OutputWriter::Meta{s.num, s.R, s.C, s.wake_nodes, t};
  std::lock_guard<std::mutex> g(w->m);
  w->q.push_back(w->next);
  w->next ^= 1;
  w->cv.notify_all();
  return ok();
}

Error output_flush(OutputWriter* w) {
  std::unique_lock<std::mutex> lk(w->m);
  w->cv.wait(lk, [&] { return w->q.empty(); });
  for (FILE* f : w->files)
    if (f) fflush(f);
  return w->err.empty() ? ok() : fail(kErrInvalid, w->err);
}

Error output_close(OutputWriter* w) {
  if (!w) return ok();
  Error e = output_flush(w);
  {
    std::lock_guard<std::mutex> g(w->m);
    w->stop = true;
    w->cv.notify_all();
  }
  w->th.join();
  for (FILE* f : w->files)
    if (f && fclose(f) != 0 && !e.code) e = fail(kErrInvalid, "output close failed");
  for (auto& s : w->slot) {
    cudaFree(s.d);
    cudaFreeHost(s.h);
    if (s.ready) cudaEventDestroy(s.ready);
    if (s.copied) cudaEventDestroy(s.copied);
  }
  if (w->os) cudaStreamDestroy(w->os);
  delete w;
  return e;
}

}  // namespace uvlm
