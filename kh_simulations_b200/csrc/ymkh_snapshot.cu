// ymkh_snapshot.cu — state snapshots written by host threads.
//
// The reference copies 25 arrays to the host after a step and hands them to
// a std::thread that writes a 26-column CSV, keeping at most four writers
// and joining the oldest first (ymgpu2d/main_ym.cu:260-313).  Here the copies
// are enqueued on the caller's stream into a pinned buffer, an event marks
// their end, and the writer thread waits on that event: the caller's stream
// is never synchronised, and the step loop continues while the file is
// formatted.  The CSV is the reference's byte for byte: its values are
// printed by an ostream of default precision, which is printf "%g", and
// std::to_chars(general, 6) gives that same text.  The FP64 form stores the
// state exactly.

#include <charconv>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "ymkh_common.cuh"

namespace ymkh {

namespace {

constexpr int A0 = YMKH_NFIELDS;                 // fluid A arrays start
constexpr int B0 = YMKH_NFIELDS + YMKH_NFLUID;  // fluid B arrays start

// Column order of ymgpu2d/main_ym.cu:291-306, as state indices.
constexpr int kCsvCols[24] = {BY1,      BY2,      BY3,      AZ2,      AZ3,      A0 + FPZ, A0 + FPX, A0 + FQ1,
                              B0 + FPZ, B0 + FPX, B0 + FQ1, EX1,      EX2,      EX3,      EZ1,      EZ2,
                              EZ3,      A0 + FN,  B0 + FN,  A0 + FQ2, A0 + FQ3, B0 + FQ2, B0 + FQ3, AZ1};
constexpr char kCsvHeader[] =
    "X,Z,By1,By2,By3,Az2,Az3,PzA,PxA,Q1A,PzB,PxB,Q1B,Ex1,Ex2,Ex3,Ez1,Ez2,Ez3,nA,nB,Q2A,Q3A,Q2B,Q3B,Az1\n";

constexpr int kMaxWriters = 4;
constexpr size_t kMaxPinnedInFlight = size_t(8) << 30;  // bytes of staged state held by writers at once
constexpr size_t kChunk = size_t(4) << 20;

struct Job {
  std::thread th;
  double* host = nullptr;  // pinned copy of the 24 arrays, state order
  size_t bytes = 0;
  cudaEvent_t copied = nullptr;
  int rc = 0;
  std::string err;
};

inline char* put_g6(char* p, double v) {
  return std::to_chars(p, p + 32, v, std::chars_format::general, 6).ptr;
}

int write_csv(const std::string& path, const double* h, int nx, int nz, double dx, double dz, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path;
    return YMKH_EINVAL;
  }
  const size_t N = (size_t)nx * (size_t)nz;
  std::vector<char> buf(kChunk + 27 * 32);
  size_t used = 0;
  bool ok = std::fwrite(kCsvHeader, 1, sizeof kCsvHeader - 1, f) == sizeof kCsvHeader - 1;
  for (int z = 0; z < nz && ok; ++z) {
    for (int x = 0; x < nx; ++x) {
      const size_t i = (size_t)x + (size_t)z * (size_t)nx;
      char* p = buf.data() + used;
      p = put_g6(p, x * dx);
      *p++ = ',';
      p = put_g6(p, z * dz);
      for (int k = 0; k < 24; ++k) {
        *p++ = ',';
        p = put_g6(p, h[(size_t)kCsvCols[k] * N + i]);
      }
      *p++ = '\n';
      used = (size_t)(p - buf.data());
      if (used >= kChunk) {
        ok = std::fwrite(buf.data(), 1, used, f) == used;
        used = 0;
        if (!ok) break;
      }
    }
  }
  if (ok && used) ok = std::fwrite(buf.data(), 1, used, f) == used;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    err = "write failed: " + path;
    return YMKH_EINVAL;
  }
  return 0;
}

int write_fp64(const std::string& path, const double* h, int nx, int nz, double dx, double dz, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path;
    return YMKH_EINVAL;
  }
  unsigned char hdr[40];
  const uint32_t meta[4] = {1u, (uint32_t)nx, (uint32_t)nz, (uint32_t)YMKH_NSTATE};
  std::memcpy(hdr, "YMKHSNP1", 8);
  std::memcpy(hdr + 8, meta, 16);
  std::memcpy(hdr + 24, &dx, 8);
  std::memcpy(hdr + 32, &dz, 8);
  const size_t n = (size_t)YMKH_NSTATE * (size_t)nx * (size_t)nz;
  bool ok = std::fwrite(hdr, 1, sizeof hdr, f) == sizeof hdr;
  ok = ok && std::fwrite(h, sizeof(double), n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    err = "write failed: " + path;
    return YMKH_EINVAL;
  }
  return 0;
}

}  // namespace

class SnapshotQueue {
 public:
  explicit SnapshotQueue(int device) : device_(device) {}
  ~SnapshotQueue() {
    std::string e;
    wait(e);
    for (auto& b : free_) cudaFreeHost(b.first);
  }

  int submit(const State& st, int nx, int nz, double dx, double dz, const char* path, int format, cudaStream_t s,
             std::string& err) {
    const size_t N = (size_t)nx * (size_t)nz;
    const size_t bytes = (size_t)YMKH_NSTATE * N * sizeof(double);
    while (!active_.empty() && ((int)active_.size() >= kMaxWriters || in_flight_ + bytes > kMaxPinnedInFlight)) reap();
    if (first_rc_) return take_error(err);
    Job* j = new Job;
    j->bytes = bytes;
    j->host = take_buffer(bytes);
    if (!j->host) {
      delete j;
      err = "pinned host buffer for a snapshot";
      return YMKH_ENOMEM;
    }
    cudaError_t e = cudaEventCreateWithFlags(&j->copied, cudaEventDisableTiming);
    const double* const* src[3] = {st.f, st.a, st.b};
    for (int k = 0; k < YMKH_NSTATE && e == cudaSuccess; ++k) {
      const double* p = k < A0 ? src[0][k] : (k < B0 ? src[1][k - A0] : src[2][k - B0]);
      e = cudaMemcpyAsync(j->host + (size_t)k * N, p, N * sizeof(double), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaEventRecord(j->copied, s);
    if (e != cudaSuccess) {
      // copies already enqueued must land before the buffer is reused
      cudaStreamSynchronize(s);
      if (j->copied) cudaEventDestroy(j->copied);
      give_buffer(j->host, bytes);
      delete j;
      err = std::string("snapshot copies: ") + cudaGetErrorString(e);
      return YMKH_ECUDA;
    }
    std::string p(path);
    const int dev = device_;
    j->th = std::thread([j, dev, p, format, nx, nz, dx, dz]() {
      cudaSetDevice(dev);
      cudaError_t ce = cudaEventSynchronize(j->copied);
      if (ce != cudaSuccess) {
        j->rc = YMKH_ECUDA;
        j->err = std::string("snapshot copies: ") + cudaGetErrorString(ce);
        return;
      }
      j->rc = format == YMKH_SNAP_CSV ? write_csv(p, j->host, nx, nz, dx, dz, j->err)
                                      : write_fp64(p, j->host, nx, nz, dx, dz, j->err);
    });
    in_flight_ += bytes;
    active_.push_back(j);
    return 0;
  }

  int wait(std::string& err) {
    while (!active_.empty()) reap();
    return take_error(err);
  }

 private:
  void reap() {
    Job* j = active_.front();
    active_.pop_front();
    j->th.join();
    if (j->rc && !first_rc_) {
      first_rc_ = j->rc;
      first_err_ = j->err;
    }
    cudaEventDestroy(j->copied);
    in_flight_ -= j->bytes;
    give_buffer(j->host, j->bytes);
    delete j;
  }
  int take_error(std::string& err) {
    const int rc = first_rc_;
    if (rc) err = first_err_;
    first_rc_ = 0;
    first_err_.clear();
    return rc;
  }
  double* take_buffer(size_t bytes) {
    for (size_t i = 0; i < free_.size(); ++i)
      if (free_[i].second == bytes) {
        double* p = free_[i].first;
        free_.erase(free_.begin() + (long)i);
        return p;
      }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return (double*)p;
  }
  void give_buffer(double* p, size_t bytes) {
    free_.push_back({p, bytes});
    while ((int)free_.size() > kMaxWriters) {
      cudaFreeHost(free_.front().first);
      free_.erase(free_.begin());
    }
  }

  int device_;
  std::deque<Job*> active_;
  std::vector<std::pair<double*, size_t>> free_;
  size_t in_flight_ = 0;
  int first_rc_ = 0;
  std::string first_err_;
};

SnapshotQueue* snapshot_queue_create(int device) { return new SnapshotQueue(device); }
void snapshot_queue_destroy(SnapshotQueue* q) { delete q; }
int snapshot_submit(SnapshotQueue* q, const State& st, int nx, int nz, double dx, double dz, const char* path,
                    int format, cudaStream_t s, std::string& err) {
  return q->submit(st, nx, nz, dx, dz, path, format, s, err);
}
int snapshot_wait(SnapshotQueue* q, std::string& err) { return q->wait(err); }

}  // namespace ymkh
