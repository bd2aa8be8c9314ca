// io.h -- host interface between the context (api.cu) and the writers and
// reader of the reference's output and reload files (io.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "device_state.h"

namespace gg {

// Per-particle attributes that reload files carry and the step does not use
// (Particle::write2014, Particle.cpp:1146-1157), by upload index.
struct RecordAttr {
  int geom_type;       // m_GeomType: index of the reference particle type
  int tag;             // 0 interior, 1 buffer zone, 2 clone
  int active;          // m_activity == COMPUTE
  int transform_type;  // Transform::m_type bits (Transform.hh:246-260)
};

// What the writers read of a context: the current particle arrays (slot
// order; orig maps a slot to its upload index), the latest contact memory
// (rows by upload index) and the tables that name particles and obstacles.
// Every pointer is device memory.
struct IoView {
  int precision;
  cudaStream_t stream;
  int n;
  const double4* xr;
  const double4* q;
  const double* basis;  // nullptr: the rotation matrix of the quaternion
  const void* v;
  const void* w;
  const void* F;
  const void* T;
  const int4* meta;  // id, material, shape, system
  const int* orig;
  const int* coord;  // by slot
  const void* hist;  // HistEntry<R>, row = upload index
  const int* hist_n;
  int hist_cap;
  const int* row_id;                   // particle id by upload index
  const int* row_sys;                  // system by upload index
  const unsigned long long* row_keys;  // sorted (system, id) keys ...
  const int* key_rows;                 // ... and their upload indices
  const int* obs_id;                   // global obstacle index -> obstacle id
  const int* sys_obs_offset;           // first global obstacle index of each system
  const RecordAttr* attr;              // by upload index
  int moved;  // particles moved since their upload: transform type |= ROTATION | TRANSLATION
};

// Device scratch and pinned staging kept by the context between writes.
struct IoScratch {
  void* dev = nullptr;  // work arrays
  size_t dev_bytes = 0;
  void* out = nullptr;  // formatted bytes
  size_t out_bytes = 0;
  void* pinned[2] = {nullptr, nullptr};
  size_t pinned_bytes = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~IoScratch();
  // at least `bytes` of work space; the first `keep` bytes survive a regrowth
  char* work(size_t bytes, size_t keep, cudaStream_t st, std::string& err);
  char* output(size_t bytes, std::string& err);
};

// AllComponents::write particle file (AllComponents.cpp:1148-1180): text
// (Particle::write2014 lines) or hybrid binary (byte count, write2014_binary)
int write_reload_particles(const IoView& v, IoScratch& s, const char* path, int binary, int64_t* bytes,
                           std::string& err);

// RawDataPostProcessingWriter::one_output_Standard (RawDataPostProcessingWriter.cpp:369-600)
int write_rawdata(const IoView& v, IoScratch& s, const char* root, double time, int system, int n_total,
                  int binary, int truncate, int64_t* bytes, std::string& err);

// A particle file read back (Particle::read2014 / read2014_binary,
// Particle.cpp:972-1072): per particle, in file order, the record fields, and
// every contact-map entry (Component::readContactMap2014(_binary),
// Component.cpp:858-907) with its holder's id.
struct ReloadData {
  std::vector<int> geom_type, id, tag, active, transform_type;
  std::vector<double> position, basis, velocity, quaternion, omega, force, torque;  // quaternion: x y z w
  std::vector<int> owner, other;
  std::vector<double> kdelta, prev_normal, spring_torque;
};

int read_reload_particles(const char* path, int binary, ReloadData& out, std::string& err);

// the device formatter over n host values, one per line (a check of the formatter)
int format_doubles(const double* x, int64_t n, int P, char* out, int64_t cap, int64_t* length, std::string& err);

}  // namespace gg
