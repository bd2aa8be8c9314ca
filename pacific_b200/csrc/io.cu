// io.cu -- the reference's particle reload file and RawData time series,
// formatted on the device.
//
//   AllComponents::write, particle file   Component/src/AllComponents.cpp:1148-1180
//   Particle::write2014 / write2014_binary Component/src/Particle.cpp:1146-1195, get_numberOfBytes :1201-1208
//   Transform::writeTransform2014(_binary) Geometry/src/Transform.cpp:416-440
//   ParticleKinematics::writeParticleKinematics2014(_binary) Component/src/ParticleKinematics.cpp:331-355
//   SecondOrderLeapFrog::writeParticleKinematics2014(_binary) TimeIntegration/src/SecondOrderLeapFrog.cpp:102-122
//   Component::writeContactMemory2014(_binary) Component/src/Component.cpp:776-835
//   RawDataPostProcessingWriter::one_output_Standard PostProcessing/src/RawDataPostProcessingWriter.cpp:369-600
//
// Layout of a write: the contact memory, kept once per pair at the lower id,
// is expanded into the per-particle maps of the reference (both sides of every
// pair, the partner's entry negated, Component.cpp:675-684), each sorted by
// the map key (1, partner id, 1); a first pass measures every record's text,
// an exclusive scan places the records, a second pass formats them in place;
// the bytes stream to the host through two pinned staging buffers while the
// host writes the previous chunk.  Values outside the device formatter's range
// (format.cuh) make the host format the whole file from downloaded arrays with
// the same record code.
#include "io.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/grains_gpu.h"
#include "format.cuh"

namespace gg {

IoScratch::~IoScratch() {
  if (dev) cudaFree(dev);
  if (out) cudaFree(out);
  for (int k = 0; k < 2; ++k) {
    if (pinned[k]) cudaFreeHost(pinned[k]);
    if (ev[k]) cudaEventDestroy(ev[k]);
  }
}

char* IoScratch::work(size_t bytes, size_t keep, cudaStream_t st, std::string& err) {
  if (bytes > dev_bytes) {
    void* p = nullptr;
    const size_t want = bytes + bytes / 4;
    if (cudaMalloc(&p, want) != cudaSuccess) {
      err = "device scratch allocation failed";
      return nullptr;
    }
    if (dev && keep) cudaMemcpyAsync(p, dev, std::min(keep, dev_bytes), cudaMemcpyDeviceToDevice, st);
    if (dev) {
      cudaStreamSynchronize(st);
      cudaFree(dev);
    }
    dev = p;
    dev_bytes = want;
  }
  return (char*)dev;
}

char* IoScratch::output(size_t bytes, std::string& err) {
  if (bytes > out_bytes) {
    if (out) cudaFree(out);
    out = nullptr;
    out_bytes = 0;
    const size_t want = bytes + bytes / 4 + 4096;
    if (cudaMalloc(&out, want) != cudaSuccess) {
      err = "device output allocation failed";
      return nullptr;
    }
    out_bytes = want;
  }
  return (char*)out;
}

namespace {

constexpr int kScanBlock = 1024;
constexpr int kThreads = 256;

// one contact-map entry of a particle: key (1, other, 1), value (active,
// kdelta, previous normal, rolling spring torque)
struct Ent {
  int other;
  int pad;
  double v[9];
};

// ---- exclusive scan of int64 (n + 1 entries: the last one receives the total)
__global__ void scan_block_kernel(int64_t* a, int64_t* sums, int64_t n) {
  __shared__ int64_t sh[kScanBlock];
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const int64_t x = i < n ? a[i] : 0;
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int off = 1; off < kScanBlock; off <<= 1) {
    const int64_t y = threadIdx.x >= (unsigned)off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += y;
    __syncthreads();
  }
  if (i < n) a[i] = sh[threadIdx.x] - x;
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void add_block_offsets_kernel(int64_t* a, const int64_t* offs, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) a[i] += offs[blockIdx.x];
}

size_t scan_scratch(int64_t n) {
  size_t total = 0;
  for (int64_t m = n; m > 1;) {
    m = (m + kScanBlock - 1) / kScanBlock;
    total += (size_t)m + 64;
  }
  return total * sizeof(int64_t);
}

void exclusive_scan(int64_t* a, int64_t n, int64_t* tmp, cudaStream_t st) {
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  scan_block_kernel<<<(unsigned)nb, kScanBlock, 0, st>>>(a, tmp, n);
  if (nb > 1) {
    exclusive_scan(tmp, nb, tmp + nb + 64, st);
    add_block_offsets_kernel<<<(unsigned)nb, kScanBlock, 0, st>>>(a, tmp, n);
  }
}

// order-preserving key of (system, id)
GG_HD unsigned long long row_key(int sys, int id) {
  return ((unsigned long long)(unsigned)sys << 32) | (unsigned)(id ^ (int)0x80000000);
}

__device__ int find_row(const unsigned long long* keys, const int* rows, int n, unsigned long long key) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const unsigned long long k = keys[mid];
    if (k == key) return rows[mid];
    if (k < key) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// slot of each upload index
__global__ void inverse_kernel(const int* orig, int* inv, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) inv[orig[t]] = t;
}

// incoming (partner-side) entries of every row; pr = partner row per entry
template <typename R>
__global__ void count_incoming_kernel(const HistEntry<R>* hist, const int* hist_n, int H, int n,
                                      const int* host_sys_dev, const unsigned long long* keys, const int* rows,
                                      int* pr, int64_t* in_cnt, int* bad) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int c = hist_n[r];
  for (int k = 0; k < c; ++k) {
    const HistEntry<R>& e = hist[(size_t)r * H + k];
    int p = -1;
    if (!(e.flags & 1)) {
      p = find_row(keys, rows, n, row_key(host_sys_dev[r], e.other));
      if (p < 0) atomicOr(bad, 2);
      else atomicAdd((unsigned long long*)&in_cnt[p], 1ull);
    }
    pr[(size_t)r * H + k] = p;
  }
}

__global__ void entry_totals_kernel(const int* hist_n, int64_t* cnt, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) cnt[r] += hist_n[r];
}

template <typename R>
__global__ void fill_entries_kernel(const HistEntry<R>* hist, const int* hist_n, int H, int n, const int* pr,
                                    const int* host_id_dev, const int* host_sys_dev, const int* obs_id,
                                    const int* sys_obs_offset, const int64_t* eoff, int* fill, Ent* ents) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int c = hist_n[r];
  const int64_t base = eoff[r];
  for (int k = 0; k < c; ++k) {
    const HistEntry<R>& e = hist[(size_t)r * H + k];
    Ent x;
    x.pad = 0;
    x.other = (e.flags & 1) ? obs_id[sys_obs_offset[host_sys_dev[r]] + e.other] : e.other;
    for (int t = 0; t < 3; ++t) {
      x.v[t] = (double)e.kd[t];
      x.v[3 + t] = (double)e.n[t];
      x.v[6 + t] = (double)e.sp[t];
    }
    ents[base + k] = x;
    const int p = pr[(size_t)r * H + k];
    if (p >= 0) {
      Ent y;
      y.pad = 0;
      y.other = host_id_dev[r];
      for (int t = 0; t < 9; ++t) y.v[t] = -x.v[t];
      const int j = atomicAdd(&fill[p], 1);
      ents[eoff[p] + hist_n[p] + j] = y;
    }
  }
}

// std::map order of the key (1, other, 1)
__global__ void sort_entries_kernel(Ent* ents, const int64_t* eoff, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  Ent* e = ents + eoff[r];
  const int c = (int)(eoff[r + 1] - eoff[r]);
  for (int i = 1; i < c; ++i) {
    Ent x = e[i];
    int j = i - 1;
    while (j >= 0 && e[j].other > x.other) {
      e[j + 1] = e[j];
      --j;
    }
    e[j + 1] = x;
  }
}


// ---- one particle record --------------------------------------------------
struct RowRec {
  int geom, id, tag, active;
  unsigned xtype;
  double pos[3], basis[9], v[3], q[4];  // q: x, y, z, w
  double w[3], F[3], T[3];
  const Ent* ents;
  int nent;
};

// the rotation matrix of a quaternion (spheres without a stored basis), the
// expression the particle download uses
GG_HD void quaternion_basis(const double* q, double* m) {
  const double x = q[0], y = q[1], z = q[2], w0 = q[3];
  m[0] = 1 - 2 * (y * y + z * z);
  m[1] = 2 * (x * y - w0 * z);
  m[2] = 2 * (x * z + w0 * y);
  m[3] = 2 * (x * y + w0 * z);
  m[4] = 1 - 2 * (x * x + z * z);
  m[5] = 2 * (y * z - w0 * x);
  m[6] = 2 * (x * z - w0 * y);
  m[7] = 2 * (y * z + w0 * x);
  m[8] = 1 - 2 * (x * x + y * y);
}

template <typename R>
__device__ void load_row(const IoView& V, int r, const int* inv, const Ent* ents, const int64_t* eoff, RowRec& o) {
  using V4 = typename Vec4<R>::type;
  const int t = inv[r];
  const RecordAttr at = V.attr[r];
  o.geom = at.geom_type;
  o.id = V.meta[t].x;
  o.tag = at.tag;
  o.active = at.active;
  o.xtype = (unsigned)at.transform_type | (V.moved ? 3u : 0u);
  const double4 x = V.xr[t], q = V.q[t];
  o.pos[0] = x.x; o.pos[1] = x.y; o.pos[2] = x.z;
  o.q[0] = q.x; o.q[1] = q.y; o.q[2] = q.z; o.q[3] = q.w;
  if (V.basis) {
    for (int k = 0; k < 9; ++k) o.basis[k] = V.basis[9 * (size_t)t + k];
  } else {
    quaternion_basis(o.q, o.basis);
  }
  const V4 v = ((const V4*)V.v)[t], w = ((const V4*)V.w)[t], F = ((const V4*)V.F)[t], T = ((const V4*)V.T)[t];
  o.v[0] = v.x; o.v[1] = v.y; o.v[2] = v.z;
  o.w[0] = w.x; o.w[1] = w.y; o.w[2] = w.z;
  o.F[0] = F.x; o.F[1] = F.y; o.F[2] = F.z;
  o.T[0] = T.x; o.T[1] = T.y; o.T[2] = T.z;
  o.ents = ents + eoff[r];
  o.nent = (int)(eoff[r + 1] - eoff[r]);
}

// output sinks: count only, or write at p
struct CountOut {
  int64_t len = 0;
  bool ok = true;
  GG_HD void ch(char) { ++len; }
  GG_HD void str(const char*, int n) { len += n; }
  GG_HD void raw(const void*, int n) { len += n; }
};

struct BufOut {
  char* p;
  int64_t len = 0;
  bool ok = true;
  GG_HD void ch(char c) { p[len++] = c; }
  GG_HD void str(const char* s, int n) {
    for (int i = 0; i < n; ++i) p[len + i] = s[i];
    len += n;
  }
  GG_HD void raw(const void* s, int n) { str((const char*)s, n); }
};

// GrainsExec::doubleToString(ios::scientific, P, x)
template <class O>
GG_HD void put_double(O& o, double x, int P) {
  char b[40];
#ifdef __CUDA_ARCH__
  const int k = fmt::grains_double(x, P, b);
#else
  const int k = fmt::grains_double_host(x, P, b, sizeof(b));
#endif
  if (k < 0) {
    o.ok = false;
    return;
  }
  o.str(b, k);
}

template <class O>
GG_HD void put_int(O& o, int x) {
  char b[12];
  o.str(b, fmt::int32(x, b));
}

// Group3::writeGroup3 (Geometry/src/Group3.cpp:351-359): three values, one space apart
template <class O>
GG_HD void put_group3(O& o, const double* g) {
  put_double(o, g[0], 16);
  o.ch(' ');
  put_double(o, g[1], 16);
  o.ch(' ');
  put_double(o, g[2], 16);
}

// Particle::write2014 (Particle.cpp:1146-1157): one line per particle
template <class O>
GG_HD void reload_text_record(O& o, const RowRec& r) {
  put_int(o, r.geom);
  o.ch(' ');
  put_int(o, r.id);
  o.ch(' ');
  put_int(o, r.tag);
  o.ch(' ');
  put_int(o, r.active ? 1 : 0);
  o.ch(' ');
  // Transform::writeTransform2014: origin, Matrix::writeMatrix2014 (rows), type
  put_group3(o, r.pos);
  o.ch(' ');
  put_group3(o, r.basis);
  o.ch(' ');
  put_group3(o, r.basis + 3);
  o.ch(' ');
  put_group3(o, r.basis + 6);
  o.ch(' ');
  put_int(o, (int)r.xtype);
  o.ch(' ');
  // ParticleKinematics::writeParticleKinematics2014: v, q (w then vector), omega
  put_group3(o, r.v);
  o.ch(' ');
  put_double(o, r.q[3], 16);
  o.ch(' ');
  put_group3(o, r.q);
  o.ch(' ');
  put_group3(o, r.w);
  // SecondOrderLeapFrog::writeParticleKinematics2014: force, torque
  o.ch(' ');
  put_group3(o, r.F);
  o.ch(' ');
  put_group3(o, r.T);
  // Component::writeContactMemory2014: size, then (1, other, 1, active, kdelta, normal, spring)
  o.ch(' ');
  put_int(o, r.nent);
  for (int k = 0; k < r.nent; ++k) {
    const Ent& e = r.ents[k];
    o.ch(' ');
    o.ch('1');
    o.ch(' ');
    put_int(o, e.other);
    o.ch(' ');
    o.ch('1');
    o.ch(' ');
    o.ch('1');
    o.ch(' ');
    put_group3(o, e.v);
    o.ch(' ');
    put_group3(o, e.v + 3);
    o.ch(' ');
    put_group3(o, e.v + 6);
  }
  o.ch('\n');
}

// bytes of Particle::write2014_binary (Particle::get_numberOfBytes, Particle.cpp:1201-1208)
GG_HD int64_t binary_record_bytes(int nent) { return 248 + 88 * (int64_t)nent; }

// the byte count (size_t) then Particle::write2014_binary (Particle.cpp:1183-1195)
template <class O>
GG_HD void reload_binary_record(O& o, const RowRec& r) {
  const uint64_t nb = (uint64_t)binary_record_bytes(r.nent);
  o.raw(&nb, 8);
  const int head[3] = {r.geom, r.id, r.tag};
  o.raw(head, 12);
  const unsigned act = r.active ? 1u : 0u;
  o.raw(&act, 4);
  o.raw(r.pos, 24);
  o.raw(r.basis, 72);
  o.raw(&r.xtype, 4);
  o.raw(r.v, 24);
  o.raw(&r.q[3], 8);
  o.raw(r.q, 24);
  o.raw(r.w, 24);
  o.raw(r.F, 24);
  o.raw(r.T, 24);
  o.raw(&r.nent, 4);
  for (int k = 0; k < r.nent; ++k) {
    const Ent& e = r.ents[k];
    const int key[4] = {1, e.other, 1, 1};
    o.raw(key, 16);
    o.raw(e.v, 72);
  }
}

template <typename R>
__global__ void reload_length_kernel(IoView V, const int* inv, const Ent* ents, const int64_t* eoff, int binary,
                                     int64_t* len, int* bad) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= V.n) return;
  RowRec rec;
  load_row<R>(V, r, inv, ents, eoff, rec);
  if (binary) {
    len[r] = binary_record_bytes(rec.nent) + 8;
    return;
  }
  CountOut o;
  reload_text_record(o, rec);
  if (!o.ok) atomicOr(bad, 1);
  len[r] = o.len;
}

template <typename R>
__global__ void reload_write_kernel(IoView V, const int* inv, const Ent* ents, const int64_t* eoff, int binary,
                                    const int64_t* off, char* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= V.n) return;
  RowRec rec;
  load_row<R>(V, r, inv, ents, eoff, rec);
  BufOut o{out + off[r]};
  if (binary) reload_binary_record(o, rec);
  else reload_text_record(o, rec);
}


// ---- RawData ------------------------------------------------------------------
// files of one output, in the reference's order (RawDataPostProcessingWriter.cpp:326-362)
constexpr int kRawFiles = 10;
const char* const kRawNames[kRawFiles] = {"_position_x.dat", "_position_y.dat", "_position_z.dat",
                                          "_translational_velocity_x.dat", "_translational_velocity_y.dat",
                                          "_translational_velocity_z.dat", "_angular_velocity_x.dat",
                                          "_angular_velocity_y.dat", "_angular_velocity_z.dat",
                                          "_coordinationNumber.dat"};

// slot of each particle id 1..n_total of one system (-1: none, or a periodic clone)
__global__ void slot_of_id_kernel(const int4* meta, const int* orig, const RecordAttr* attr, int n, int sys,
                                  int n_total, int* sid) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 m = meta[t];
  if (m.w != sys || m.x < 1 || m.x > n_total) return;
  if (attr[orig[t]].tag == 2) return;
  sid[m.x - 1] = t;
}

// value of file f (0-8) for id i: the particle's, or the inactive defaults
// (GrainsExec::m_defaultInactivePos = -1e10, zero velocities)
template <typename R>
__device__ double raw_value(const IoView& V, const int* sid, int f, int i) {
  using V4 = typename Vec4<R>::type;
  const int t = sid[i];
  if (t < 0) return f < 3 ? -1.e10 : 0.;
  if (f < 3) {
    const double4 x = V.xr[t];
    return f == 0 ? x.x : (f == 1 ? x.y : x.z);
  }
  const V4 u = f < 6 ? ((const V4*)V.v)[t] : ((const V4*)V.w)[t];
  const int c = f % 3;
  return c == 0 ? (double)u.x : (c == 1 ? (double)u.y : (double)u.z);
}

// record j of file f's line: 0 = the time (not in the coordination file),
// 1..n_total = " value", n_total + 1 = newline
template <typename R, class O>
__device__ void raw_text_record(O& o, const IoView& V, const int* sid, int f, int j, int n_total, double time) {
  if (j == 0) {
    if (f < kRawFiles - 1) put_double(o, time, 6);
    return;
  }
  if (j == n_total + 1) {
    o.ch('\n');
    return;
  }
  o.ch(' ');
  if (f == kRawFiles - 1) {
    const int t = sid[j - 1];
    put_int(o, t < 0 ? 0 : V.coord[t]);
  } else {
    put_double(o, raw_value<R>(V, sid, f, j - 1), 6);
  }
}

// the particle type file: "type " per id (-1 when absent), then a newline
__device__ int raw_type(const IoView& V, const int* sid, int i) {
  const int t = sid[i];
  return t < 0 ? -1 : V.attr[V.orig[t]].geom_type;
}

template <typename R>
__global__ void raw_length_kernel(IoView V, const int* sid, int n_total, double time, int64_t* len, int* bad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)n_total + 2;
  if (k < kRawFiles * per) {
    CountOut o;
    raw_text_record<R>(o, V, sid, (int)(k / per), (int)(k % per), n_total, time);
    if (!o.ok) atomicOr(bad, 1);
    len[k] = o.len;
  } else if (k < kRawFiles * per + n_total + 1) {
    const int i = (int)(k - kRawFiles * per);
    CountOut o;
    if (i == n_total) {
      o.ch('\n');
    } else {
      put_int(o, raw_type(V, sid, i));
      o.ch(' ');
    }
    len[k] = o.len;
  }
}

template <typename R>
__global__ void raw_write_kernel(IoView V, const int* sid, int n_total, double time, const int64_t* off,
                                 char* out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)n_total + 2;
  if (k < kRawFiles * per) {
    BufOut o{out + off[k]};
    raw_text_record<R>(o, V, sid, (int)(k / per), (int)(k % per), n_total, time);
  } else if (k < kRawFiles * per + n_total + 1) {
    const int i = (int)(k - kRawFiles * per);
    BufOut o{out + off[k]};
    if (i == n_total) {
      o.ch('\n');
    } else {
      put_int(o, raw_type(V, sid, i));
      o.ch(' ');
    }
  }
}

// binary: per file the time (twice for the z angular velocity, as the
// reference writes it, RawDataPostProcessingWriter.cpp:397-400) then one
// double per id; coordination numbers and types as ints, without the time
template <typename R>
__global__ void raw_binary_kernel(IoView V, const int* sid, int n_total, double time, char* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_total) return;
  int64_t base = 0;
  for (int f = 0; f < kRawFiles - 1; ++f) {
    const int64_t head = f == 8 ? 16 : 8;
    double* d = (double*)(out + base + head);
    if (i == 0) {
      ((double*)(out + base))[0] = time;
      if (f == 8) ((double*)(out + base))[1] = time;
    }
    d[i] = raw_value<R>(V, sid, f, i);
    base += head + 8 * (int64_t)n_total;
  }
  const int t = sid[i];
  ((int*)(out + base))[i] = t < 0 ? 0 : V.coord[t];
  base += 4 * (int64_t)n_total;
  ((int*)(out + base))[i] = raw_type(V, sid, i);
}

// ---- host side -------------------------------------------------------------------
struct Segment {
  std::string path;
  int64_t off, len;
  bool truncate;
};

#define IO_CK(x)                                                     \
  do {                                                               \
    cudaError_t e_ = (x);                                            \
    if (e_ != cudaSuccess) {                                         \
      err = std::string(#x) + ": " + cudaGetErrorString(e_);         \
      return GRAINS_GPU_CUDA_ERROR;                                  \
    }                                                                \
  } while (0)

constexpr size_t kChunk = 32u << 20;

// device bytes -> files, through two pinned staging buffers: the copy of the
// next chunk overlaps the host's write of the current one
int stream_out(IoScratch& s, cudaStream_t st, const char* dev, const std::vector<Segment>& segs, std::string& err) {
  if (!s.pinned[0]) {
    for (int k = 0; k < 2; ++k) {
      IO_CK(cudaMallocHost(&s.pinned[k], kChunk));
      IO_CK(cudaEventCreateWithFlags(&s.ev[k], cudaEventDisableTiming));
    }
    s.pinned_bytes = kChunk;
  }
  struct Piece {
    int seg;
    int64_t off, len;
  };
  std::vector<Piece> pieces;
  for (size_t g = 0; g < segs.size(); ++g)
    for (int64_t o = 0; o < segs[g].len || (o == 0 && segs[g].len == 0); o += (int64_t)kChunk) {
      pieces.push_back({(int)g, segs[g].off + o, std::min<int64_t>((int64_t)kChunk, segs[g].len - o)});
      if (segs[g].len == 0) break;
    }
  auto issue = [&](size_t i) -> int {
    const Piece& p = pieces[i];
    if (p.len > 0) IO_CK(cudaMemcpyAsync(s.pinned[i & 1], dev + p.off, (size_t)p.len, cudaMemcpyDeviceToHost, st));
    IO_CK(cudaEventRecord(s.ev[i & 1], st));
    return 0;
  };
  FILE* f = nullptr;
  int open_seg = -1;
  int rc = pieces.empty() ? 0 : issue(0);
  for (size_t i = 0; i < pieces.size() && !rc; ++i) {
    if (i + 1 < pieces.size() && (rc = issue(i + 1))) break;
    const Piece& p = pieces[i];
    if (p.seg != open_seg) {
      if (f) std::fclose(f);
      f = std::fopen(segs[p.seg].path.c_str(), segs[p.seg].truncate ? "wb" : "ab");
      if (!f) {
        err = "cannot open " + segs[p.seg].path;
        rc = GRAINS_GPU_INVALID_ARGUMENT;
        break;
      }
      open_seg = p.seg;
    }
    if (cudaEventSynchronize(s.ev[i & 1]) != cudaSuccess) {
      err = "staging copy failed";
      rc = GRAINS_GPU_CUDA_ERROR;
      break;
    }
    if (p.len > 0 && std::fwrite(s.pinned[i & 1], 1, (size_t)p.len, f) != (size_t)p.len) {
      err = "write failed: " + segs[p.seg].path;
      rc = GRAINS_GPU_INVALID_ARGUMENT;
      break;
    }
  }
  if (f) std::fclose(f);
  cudaStreamSynchronize(st);
  return rc;
}

unsigned blocks_for(int64_t n, int threads = kThreads) { return (unsigned)((n + threads - 1) / threads); }


size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// host copies of what the record code reads, for the fallback formatter
template <typename R>
struct HostRows {
  using V4 = typename Vec4<R>::type;
  std::vector<double4> xr, q;
  std::vector<double> basis;
  std::vector<V4> v, w, F, T;
  std::vector<int4> meta;
  std::vector<int> inv;
  std::vector<RecordAttr> attr;
  std::vector<Ent> ents;
  std::vector<int64_t> eoff;
  int moved = 0;

  int fetch(const IoView& V, const int* d_inv, const Ent* d_ents, const int64_t* d_eoff, int64_t E,
            std::string& err) {
    const int n = V.n;
    xr.resize(n); q.resize(n); v.resize(n); w.resize(n); F.resize(n); T.resize(n); meta.resize(n);
    inv.resize(n); attr.resize(n); ents.resize((size_t)E); eoff.resize((size_t)n + 1);
    if (V.basis) basis.resize(9 * (size_t)n);
    cudaStream_t st = V.stream;
    IO_CK(cudaMemcpyAsync(xr.data(), V.xr, n * sizeof(double4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(q.data(), V.q, n * sizeof(double4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(v.data(), V.v, n * sizeof(V4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(w.data(), V.w, n * sizeof(V4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(F.data(), V.F, n * sizeof(V4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(T.data(), V.T, n * sizeof(V4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(meta.data(), V.meta, n * sizeof(int4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(inv.data(), d_inv, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(attr.data(), V.attr, n * sizeof(RecordAttr), cudaMemcpyDeviceToHost, st));
    if (E) IO_CK(cudaMemcpyAsync(ents.data(), d_ents, (size_t)E * sizeof(Ent), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(eoff.data(), d_eoff, ((size_t)n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    if (V.basis) IO_CK(cudaMemcpyAsync(basis.data(), V.basis, 9 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaStreamSynchronize(st));
    moved = V.moved;
    return 0;
  }

  void load(int r, RowRec& o) const {
    const int t = inv[r];
    const RecordAttr at = attr[r];
    o.geom = at.geom_type;
    o.id = meta[t].x;
    o.tag = at.tag;
    o.active = at.active;
    o.xtype = (unsigned)at.transform_type | (moved ? 3u : 0u);
    o.pos[0] = xr[t].x; o.pos[1] = xr[t].y; o.pos[2] = xr[t].z;
    o.q[0] = q[t].x; o.q[1] = q[t].y; o.q[2] = q[t].z; o.q[3] = q[t].w;
    if (!basis.empty()) {
      for (int k = 0; k < 9; ++k) o.basis[k] = basis[9 * (size_t)t + k];
    } else {
      quaternion_basis(o.q, o.basis);
    }
    o.v[0] = v[t].x; o.v[1] = v[t].y; o.v[2] = v[t].z;
    o.w[0] = w[t].x; o.w[1] = w[t].y; o.w[2] = w[t].z;
    o.F[0] = F[t].x; o.F[1] = F[t].y; o.F[2] = F[t].z;
    o.T[0] = T[t].x; o.T[1] = T[t].y; o.T[2] = T[t].z;
    o.ents = ents.data() + eoff[r];
    o.nent = (int)(eoff[r + 1] - eoff[r]);
  }
};

// runs f(begin, end) over [0, n) on the host's cores
template <class F>
void parallel_rows(int64_t n, F f) {
  const int nt = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (n < 4096 || nt == 1) {
    f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  for (int k = 0; k < nt; ++k) {
    const int64_t b = n * k / nt, e = n * (k + 1) / nt;
    th.emplace_back([=] { f(b, e); });
  }
  for (auto& t : th) t.join();
}

int write_host_buffer(const std::vector<Segment>& segs, const std::vector<char>& buf, std::string& err) {
  for (const Segment& g : segs) {
    FILE* f = std::fopen(g.path.c_str(), g.truncate ? "wb" : "ab");
    if (!f) {
      err = "cannot open " + g.path;
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    const bool ok = g.len == 0 || std::fwrite(buf.data() + g.off, 1, (size_t)g.len, f) == (size_t)g.len;
    std::fclose(f);
    if (!ok) {
      err = "write failed: " + g.path;
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
  }
  return 0;
}

template <typename R>
int write_reload_t(const IoView& V, IoScratch& S, const char* path, int binary, int64_t* bytes, std::string& err) {
  const int n = V.n, H = V.hist_cap;
  cudaStream_t st = V.stream;
  const size_t o_inv = 0, o_pr = al256(o_inv + 4 * (size_t)n), o_eoff = al256(o_pr + 4 * (size_t)n * H),
               o_fill = al256(o_eoff + 8 * ((size_t)n + 1)), o_bad = al256(o_fill + 4 * (size_t)n),
               o_tmp = al256(o_bad + 16), o_end1 = al256(o_tmp + scan_scratch((int64_t)n + 1));
  char* w = S.work(o_end1, 0, st, err);
  if (!w) return GRAINS_GPU_CUDA_ERROR;
  IO_CK(cudaMemsetAsync(w + o_eoff, 0, 8 * ((size_t)n + 1), st));
  IO_CK(cudaMemsetAsync(w + o_fill, 0, 4 * (size_t)n, st));
  IO_CK(cudaMemsetAsync(w + o_bad, 0, 16, st));
  const unsigned nb = blocks_for(n);
  inverse_kernel<<<nb, kThreads, 0, st>>>(V.orig, (int*)(w + o_inv), n);
  count_incoming_kernel<R><<<nb, kThreads, 0, st>>>((const HistEntry<R>*)V.hist, V.hist_n, H, n, V.row_sys,
                                                    V.row_keys, V.key_rows, (int*)(w + o_pr),
                                                    (int64_t*)(w + o_eoff), (int*)(w + o_bad));
  entry_totals_kernel<<<nb, kThreads, 0, st>>>(V.hist_n, (int64_t*)(w + o_eoff), n);
  exclusive_scan((int64_t*)(w + o_eoff), (int64_t)n + 1, (int64_t*)(w + o_tmp), st);
  int64_t E = 0;
  int hbad = 0;
  IO_CK(cudaMemcpyAsync(&E, w + o_eoff + 8 * (size_t)n, 8, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaMemcpyAsync(&hbad, w + o_bad, 4, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaStreamSynchronize(st));
  IO_CK(cudaGetLastError());
  if (hbad & 2) {
    err = "contact memory names a particle id that is not uploaded";
    return GRAINS_GPU_INVALID_ARGUMENT;
  }
  const size_t o_ents = o_end1, o_len = al256(o_ents + sizeof(Ent) * (size_t)E),
               o_end2 = al256(o_len + 8 * ((size_t)n + 1));
  w = S.work(o_end2, o_end1, st, err);
  if (!w) return GRAINS_GPU_CUDA_ERROR;
  int* inv = (int*)(w + o_inv);
  const int64_t* eoff = (const int64_t*)(w + o_eoff);
  Ent* ents = (Ent*)(w + o_ents);
  int64_t* len = (int64_t*)(w + o_len);
  fill_entries_kernel<R><<<nb, kThreads, 0, st>>>((const HistEntry<R>*)V.hist, V.hist_n, H, n, (const int*)(w + o_pr),
                                                  V.row_id, V.row_sys, V.obs_id, V.sys_obs_offset, eoff,
                                                  (int*)(w + o_fill), ents);
  sort_entries_kernel<<<nb, kThreads, 0, st>>>(ents, eoff, n);
  IO_CK(cudaMemsetAsync(len + n, 0, 8, st));
  reload_length_kernel<R><<<nb, kThreads, 0, st>>>(V, inv, ents, eoff, binary, len, (int*)(w + o_bad));
  exclusive_scan(len, (int64_t)n + 1, (int64_t*)(w + o_tmp), st);
  int64_t total = 0;
  IO_CK(cudaMemcpyAsync(&total, len + n, 8, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaMemcpyAsync(&hbad, w + o_bad, 4, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaStreamSynchronize(st));
  IO_CK(cudaGetLastError());
  *bytes = total;
  std::vector<Segment> segs{{path, 0, total, true}};
  if (hbad & 1) {
    // a value outside the device formatter's range: format on the host
    HostRows<R> h;
    if (int rc = h.fetch(V, inv, ents, eoff, E, err)) return rc;
    std::vector<int64_t> off((size_t)n + 1, 0);
    parallel_rows(n, [&](int64_t b, int64_t e) {
      RowRec rec;
      for (int64_t r = b; r < e; ++r) {
        h.load((int)r, rec);
        CountOut o;
        reload_text_record(o, rec);
        off[r + 1] = o.len;
      }
    });
    for (int r = 0; r < n; ++r) off[r + 1] += off[r];
    std::vector<char> buf((size_t)off[n]);
    parallel_rows(n, [&](int64_t b, int64_t e) {
      RowRec rec;
      for (int64_t r = b; r < e; ++r) {
        h.load((int)r, rec);
        BufOut o{buf.data() + off[r]};
        reload_text_record(o, rec);
      }
    });
    *bytes = off[n];
    segs[0].len = off[n];
    return write_host_buffer(segs, buf, err);
  }
  char* out = S.output((size_t)total, err);
  if (!out) return GRAINS_GPU_CUDA_ERROR;
  reload_write_kernel<R><<<nb, kThreads, 0, st>>>(V, inv, ents, eoff, binary, len, out);
  IO_CK(cudaGetLastError());
  return stream_out(S, st, out, segs, err);
}

// host formatter of a RawData output (values outside the device formatter's range)
template <typename R>
int write_rawdata_host(const IoView& V, const int* d_sid, int n_total, double time, std::vector<Segment>& segs,
                       int64_t* bytes, std::string& err) {
  using V4 = typename Vec4<R>::type;
  const int n = V.n;
  cudaStream_t st = V.stream;
  std::vector<int> sid(n_total), coord(n), orig(n);
  std::vector<double4> xr(n);
  std::vector<V4> v(n), w(n);
  std::vector<RecordAttr> attr(n);
  if (n_total) IO_CK(cudaMemcpyAsync(sid.data(), d_sid, 4 * (size_t)n_total, cudaMemcpyDeviceToHost, st));
  if (n) {
    IO_CK(cudaMemcpyAsync(coord.data(), V.coord, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(orig.data(), V.orig, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(xr.data(), V.xr, n * sizeof(double4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(v.data(), V.v, n * sizeof(V4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(w.data(), V.w, n * sizeof(V4), cudaMemcpyDeviceToHost, st));
    IO_CK(cudaMemcpyAsync(attr.data(), V.attr, n * sizeof(RecordAttr), cudaMemcpyDeviceToHost, st));
  }
  IO_CK(cudaStreamSynchronize(st));
  auto value = [&](int f, int i) -> double {
    const int t = sid[i];
    if (t < 0) return f < 3 ? -1.e10 : 0.;
    if (f < 3) return f == 0 ? xr[t].x : (f == 1 ? xr[t].y : xr[t].z);
    const V4 u = f < 6 ? v[t] : w[t];
    const int c = f % 3;
    return c == 0 ? (double)u.x : (c == 1 ? (double)u.y : (double)u.z);
  };
  std::vector<char> buf;
  char b[64];
  auto put = [&](const char* s, int k) { buf.insert(buf.end(), s, s + k); };
  for (int f = 0; f < kRawFiles; ++f) {
    segs[f].off = (int64_t)buf.size();
    if (f < kRawFiles - 1) put(b, fmt::grains_double_host(time, 6, b, sizeof(b)));
    for (int i = 0; i < n_total; ++i) {
      buf.push_back(' ');
      if (f == kRawFiles - 1) put(b, fmt::int32(sid[i] < 0 ? 0 : coord[sid[i]], b));
      else put(b, fmt::grains_double_host(value(f, i), 6, b, sizeof(b)));
    }
    buf.push_back('\n');
    segs[f].len = (int64_t)buf.size() - segs[f].off;
  }
  segs[kRawFiles].off = (int64_t)buf.size();
  for (int i = 0; i < n_total; ++i) {
    put(b, fmt::int32(sid[i] < 0 ? -1 : attr[orig[sid[i]]].geom_type, b));
    buf.push_back(' ');
  }
  buf.push_back('\n');
  segs[kRawFiles].len = (int64_t)buf.size() - segs[kRawFiles].off;
  *bytes = (int64_t)buf.size();
  return write_host_buffer(segs, buf, err);
}

template <typename R>
int write_rawdata_t(const IoView& V, IoScratch& S, const char* root, double time, int sys, int n_total, int binary,
                    int truncate, int64_t* bytes, std::string& err) {
  cudaStream_t st = V.stream;
  const std::string base(root);
  const int64_t per = (int64_t)n_total + 2, nrec = kRawFiles * per + n_total + 1;
  const size_t o_sid = 0, o_len = al256(4 * (size_t)n_total), o_bad = al256(o_len + 8 * ((size_t)nrec + 1)),
               o_tmp = al256(o_bad + 16), o_end = al256(o_tmp + scan_scratch(nrec + 1));
  char* w = S.work(binary ? al256(4 * (size_t)n_total) : o_end, 0, st, err);
  if (!w) return GRAINS_GPU_CUDA_ERROR;
  int* sid = (int*)(w + o_sid);
  IO_CK(cudaMemsetAsync(sid, 0xff, 4 * (size_t)n_total, st));
  if (V.n) slot_of_id_kernel<<<blocks_for(V.n), kThreads, 0, st>>>(V.meta, V.orig, V.attr, V.n, sys, n_total, sid);
  std::vector<Segment> segs;
  if (binary) {
    const int64_t total = 9 * (8 + 8 * (int64_t)n_total) + 8 + 8 * (int64_t)n_total;
    char* out = S.output((size_t)total, err);
    if (!out) return GRAINS_GPU_CUDA_ERROR;
    if (n_total) raw_binary_kernel<R><<<blocks_for(n_total), kThreads, 0, st>>>(V, sid, n_total, time, out);
    else IO_CK(cudaMemcpyAsync(out, &time, 8, cudaMemcpyHostToDevice, st));
    IO_CK(cudaGetLastError());
    int64_t off = 0;
    for (int f = 0; f < kRawFiles; ++f) {
      const int64_t len = f < 9 ? (f == 8 ? 16 : 8) + 8 * (int64_t)n_total : 4 * (int64_t)n_total;
      segs.push_back({base + kRawNames[f], off, len, truncate != 0});
      off += len;
    }
    segs.push_back({base + "_particleType.dat", off, 4 * (int64_t)n_total, true});
    *bytes = total;
    if (n_total == 0) {
      // the time alone (twice in the z angular velocity file)
      for (int f = 0; f < 9; ++f) segs[f] = {base + kRawNames[f], 0, f == 8 ? 0 : 8, truncate != 0};
    }
    return stream_out(S, st, out, segs, err);
  }
  int64_t* len = (int64_t*)(w + o_len);
  IO_CK(cudaMemsetAsync(w + o_bad, 0, 16, st));
  IO_CK(cudaMemsetAsync(len + nrec, 0, 8, st));
  raw_length_kernel<R><<<blocks_for(nrec), kThreads, 0, st>>>(V, sid, n_total, time, len, (int*)(w + o_bad));
  exclusive_scan(len, nrec + 1, (int64_t*)(w + o_tmp), st);
  std::vector<int64_t> off(kRawFiles + 2);
  int hbad = 0;
  for (int f = 0; f <= kRawFiles; ++f)
    IO_CK(cudaMemcpyAsync(&off[f], len + f * per, 8, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaMemcpyAsync(&off[kRawFiles + 1], len + nrec, 8, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaMemcpyAsync(&hbad, w + o_bad, 4, cudaMemcpyDeviceToHost, st));
  IO_CK(cudaStreamSynchronize(st));
  IO_CK(cudaGetLastError());
  for (int f = 0; f < kRawFiles; ++f) segs.push_back({base + kRawNames[f], off[f], off[f + 1] - off[f], truncate != 0});
  segs.push_back({base + "_particleType.dat", off[kRawFiles], off[kRawFiles + 1] - off[kRawFiles], true});
  *bytes = off[kRawFiles + 1];
  if (hbad & 1) return write_rawdata_host<R>(V, sid, n_total, time, segs, bytes, err);
  char* out = S.output((size_t)off[kRawFiles + 1], err);
  if (!out) return GRAINS_GPU_CUDA_ERROR;
  raw_write_kernel<R><<<blocks_for(nrec), kThreads, 0, st>>>(V, sid, n_total, time, len, out);
  IO_CK(cudaGetLastError());
  return stream_out(S, st, out, segs, err);
}

}  // namespace

// ---- the formatter over an array (device) -------------------------------------
namespace {

__global__ void fmt_length_kernel(const double* x, int64_t n, int P, int64_t* len, int* bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  CountOut o;
  put_double(o, x[i], P);
  o.ch('\n');
  if (!o.ok) atomicOr(bad, 1);
  len[i] = o.len;
}

__global__ void fmt_write_kernel(const double* x, int64_t n, int P, const int64_t* off, char* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  BufOut o{out + off[i]};
  put_double(o, x[i], P);
  o.ch('\n');
}

}  // namespace

int format_doubles(const double* hx, int64_t n, int P, char* out, int64_t cap, int64_t* length, std::string& err) {
  cudaStream_t st = nullptr;
  void* mem = nullptr;
  const size_t o_x = 0, o_len = al256(8 * (size_t)n), o_bad = al256(o_len + 8 * ((size_t)n + 1)),
               o_tmp = al256(o_bad + 16), o_end = al256(o_tmp + scan_scratch(n + 1));
  IO_CK(cudaMalloc(&mem, o_end));
  char* w = (char*)mem;
  int64_t* len = (int64_t*)(w + o_len);
  int rc = 0;
  int hbad = 0;
  int64_t total = 0;
  char* dout = nullptr;
  auto body = [&]() -> int {
    IO_CK(cudaMemcpy(w + o_x, hx, 8 * (size_t)n, cudaMemcpyHostToDevice));
    IO_CK(cudaMemset(w + o_bad, 0, 16));
    IO_CK(cudaMemset(len + n, 0, 8));
    if (n) fmt_length_kernel<<<blocks_for(n), kThreads, 0, st>>>((const double*)(w + o_x), n, P, len, (int*)(w + o_bad));
    exclusive_scan(len, n + 1, (int64_t*)(w + o_tmp), st);
    IO_CK(cudaMemcpy(&total, len + n, 8, cudaMemcpyDeviceToHost));
    IO_CK(cudaMemcpy(&hbad, w + o_bad, 4, cudaMemcpyDeviceToHost));
    if (hbad) {
      err = "a value is outside the device formatter's range";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    if (total > cap) {
      err = "output buffer too small";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
    IO_CK(cudaMalloc(&dout, (size_t)total + 1));
    if (n) fmt_write_kernel<<<blocks_for(n), kThreads, 0, st>>>((const double*)(w + o_x), n, P, len, dout);
    IO_CK(cudaGetLastError());
    IO_CK(cudaMemcpy(out, dout, (size_t)total, cudaMemcpyDeviceToHost));
    return 0;
  };
  rc = body();
  if (dout) cudaFree(dout);
  cudaFree(mem);
  *length = total;
  return rc;
}

// ---- reading a particle file ---------------------------------------------------
namespace {

struct Cursor {
  const char* p;
  const char* end;
  bool ok = true;
  void skip() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  }
  double dbl() {
    skip();
    char* e = nullptr;
    const double x = std::strtod(p, &e);
    if (e == p || e > end) ok = false;
    else p = e;
    return x;
  }
  long integer() {
    skip();
    char* e = nullptr;
    const long x = std::strtol(p, &e, 10);
    if (e == p || e > end) ok = false;
    else p = e;
    return x;
  }
};

// one line of Particle::write2014
bool parse_text_line(Cursor& c, ReloadData& d) {
  d.geom_type.push_back((int)c.integer());
  const int id = (int)c.integer();
  d.id.push_back(id);
  d.tag.push_back((int)c.integer());
  d.active.push_back((int)c.integer());
  for (int k = 0; k < 3; ++k) d.position.push_back(c.dbl());
  for (int k = 0; k < 9; ++k) d.basis.push_back(c.dbl());
  d.transform_type.push_back((int)c.integer());
  for (int k = 0; k < 3; ++k) d.velocity.push_back(c.dbl());
  const double qw = c.dbl();
  for (int k = 0; k < 3; ++k) d.quaternion.push_back(c.dbl());
  d.quaternion.push_back(qw);
  for (int k = 0; k < 3; ++k) d.omega.push_back(c.dbl());
  for (int k = 0; k < 3; ++k) d.force.push_back(c.dbl());
  for (int k = 0; k < 3; ++k) d.torque.push_back(c.dbl());
  const long m = c.integer();
  if (m < 0) return false;
  for (long j = 0; j < m && c.ok; ++j) {
    c.integer();  // the holder's elementary id
    const int other = (int)c.integer();
    c.integer();  // the neighbour's elementary id
    c.integer();  // active
    d.owner.push_back(id);
    d.other.push_back(other);
    for (int k = 0; k < 3; ++k) d.kdelta.push_back(c.dbl());
    for (int k = 0; k < 3; ++k) d.prev_normal.push_back(c.dbl());
    for (int k = 0; k < 3; ++k) d.spring_torque.push_back(c.dbl());
  }
  return c.ok;
}

template <typename T>
void append(std::vector<T>& a, const std::vector<T>& b) {
  a.insert(a.end(), b.begin(), b.end());
}

void append_all(ReloadData& a, const ReloadData& b) {
  append(a.geom_type, b.geom_type); append(a.id, b.id); append(a.tag, b.tag); append(a.active, b.active);
  append(a.transform_type, b.transform_type); append(a.position, b.position); append(a.basis, b.basis);
  append(a.velocity, b.velocity); append(a.quaternion, b.quaternion); append(a.omega, b.omega);
  append(a.force, b.force); append(a.torque, b.torque); append(a.owner, b.owner); append(a.other, b.other);
  append(a.kdelta, b.kdelta); append(a.prev_normal, b.prev_normal); append(a.spring_torque, b.spring_torque);
}

template <typename T>
T take(const char*& p) {
  T x;
  std::memcpy(&x, p, sizeof(T));
  p += sizeof(T);
  return x;
}

}  // namespace

int read_reload_particles(const char* path, int binary, ReloadData& out, std::string& err) {
  out = ReloadData{};
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open ") + path;
    return GRAINS_GPU_INVALID_ARGUMENT;
  }
  std::vector<char> buf;
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  buf.resize(size > 0 ? (size_t)size : 0);
  const bool ok = buf.empty() || std::fread(buf.data(), 1, buf.size(), f) == buf.size();
  std::fclose(f);
  if (!ok) {
    err = std::string("cannot read ") + path;
    return GRAINS_GPU_INVALID_ARGUMENT;
  }
  const size_t file_bytes = buf.size();
  buf.push_back('\0');  // strtod / strtol stop at the end of the text
  if (binary) {
    // byte count, then the record (AllComponents::write, AllComponents.cpp:1159-1168)
    const char* p = buf.data();
    const char* end = p + file_bytes;
    while (p < end) {
      if (end - p < 8) break;
      const uint64_t nb = take<uint64_t>(p);
      if (nb < 248 || (uint64_t)(end - p) < nb || (nb - 248) % 88 != 0) {
        err = "malformed binary particle record";
        return GRAINS_GPU_INVALID_ARGUMENT;
      }
      const char* rec_end = p + nb;
      out.geom_type.push_back(take<int>(p));
      const int id = take<int>(p);
      out.id.push_back(id);
      out.tag.push_back(take<int>(p));
      out.active.push_back((int)take<unsigned>(p));
      for (int k = 0; k < 3; ++k) out.position.push_back(take<double>(p));
      for (int k = 0; k < 9; ++k) out.basis.push_back(take<double>(p));
      out.transform_type.push_back((int)take<unsigned>(p));
      for (int k = 0; k < 3; ++k) out.velocity.push_back(take<double>(p));
      const double qw = take<double>(p);
      for (int k = 0; k < 3; ++k) out.quaternion.push_back(take<double>(p));
      out.quaternion.push_back(qw);
      for (int k = 0; k < 3; ++k) out.omega.push_back(take<double>(p));
      for (int k = 0; k < 3; ++k) out.force.push_back(take<double>(p));
      for (int k = 0; k < 3; ++k) out.torque.push_back(take<double>(p));
      const int m = take<int>(p);
      if (m < 0 || (uint64_t)m * 88 + 248 != nb) {
        err = "binary particle record size does not match its contact map";
        return GRAINS_GPU_INVALID_ARGUMENT;
      }
      for (int j = 0; j < m; ++j) {
        take<int>(p);
        const int other = take<int>(p);
        take<int>(p);
        take<int>(p);
        out.owner.push_back(id);
        out.other.push_back(other);
        for (int k = 0; k < 3; ++k) out.kdelta.push_back(take<double>(p));
        for (int k = 0; k < 3; ++k) out.prev_normal.push_back(take<double>(p));
        for (int k = 0; k < 3; ++k) out.spring_torque.push_back(take<double>(p));
      }
      p = rec_end;
    }
    return 0;
  }
  // text: one particle per line, lines parsed in parallel chunks
  std::vector<size_t> starts;
  const char* b = buf.data();
  const size_t n = file_bytes;
  for (size_t i = 0; i < n;) {
    while (i < n && (b[i] == '\n' || b[i] == ' ' || b[i] == '\r')) ++i;
    if (i >= n) break;
    starts.push_back(i);
    const void* nl = std::memchr(b + i, '\n', n - i);
    i = nl ? (size_t)((const char*)nl - b) + 1 : n;
  }
  const int64_t lines = (int64_t)starts.size();
  const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()),
                                                             (lines + 4095) / 4096));
  std::vector<ReloadData> part(nt);
  std::vector<int> bad(nt, 0);
  std::vector<std::thread> th;
  for (int k = 0; k < nt; ++k)
    th.emplace_back([&, k] {
      const int64_t l0 = lines * k / nt, l1 = lines * (k + 1) / nt;
      for (int64_t l = l0; l < l1 && !bad[k]; ++l) {
        const char* e = (const char*)std::memchr(b + starts[l], '\n', n - starts[l]);
        Cursor c{b + starts[l], e ? e : b + n};
        if (!parse_text_line(c, part[k])) bad[k] = 1;
      }
    });
  for (auto& t : th) t.join();
  for (int k = 0; k < nt; ++k)
    if (bad[k]) {
      err = "malformed particle line";
      return GRAINS_GPU_INVALID_ARGUMENT;
    }
  for (int k = 0; k < nt; ++k) append_all(out, part[k]);
  return 0;
}

int write_reload_particles(const IoView& v, IoScratch& s, const char* path, int binary, int64_t* bytes,
                           std::string& err) {
  return v.precision == GRAINS_GPU_FP64 ? write_reload_t<double>(v, s, path, binary, bytes, err)
                                        : write_reload_t<float>(v, s, path, binary, bytes, err);
}

int write_rawdata(const IoView& v, IoScratch& s, const char* root, double time, int system, int n_total, int binary,
                  int truncate, int64_t* bytes, std::string& err) {
  return v.precision == GRAINS_GPU_FP64
             ? write_rawdata_t<double>(v, s, root, time, system, n_total, binary, truncate, bytes, err)
             : write_rawdata_t<float>(v, s, root, time, system, n_total, binary, truncate, bytes, err);
}

}  // namespace gg
