// gw_convert.cu -- the reference's graph preprocessor on the device:
// convert_to_csr + compute_block (convert_if_notexists,
// src/preprocess/conversions.hpp:181-404), behind gw_convert_edgelist.
//
// The reference reads the edge list line by line (fgets, strtok, atoi) on one
// thread.  Here the text streams through the GPU in chunks of whole lines:
// the host reads chunk k+1 from the file while the device splits chunk k into
// lines (a select over newline positions), parses one line per thread and
// appends the kept edges, packed as (source << 32 | target), in file order.
// At the end the edges are grouped by source with a stable radix sort on the
// source bits only (skipped when the file was already grouped, the case the
// reference requires), and the row pointer and column array are built from
// the sorted keys; the host writes the reference's files and block range.
#include <dirent.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "gw_ctx.h"

namespace gw {

namespace {

constexpr uint32_t kMaxLine = 1023;          // fgets(s, 1024, f) reads at most 1023 bytes
constexpr size_t kChunkBytes = 64ull << 20;  // text per device round (GW_CONVERT_CHUNK_BYTES overrides)
constexpr unsigned long long kNoLine = ~0ull;

struct LineStartAt {
  const char* t;
  __device__ bool operator()(uint64_t i) const { return i == 0 || t[i - 1] == '\n'; }
};

__device__ __forceinline__ bool is_delim(char c) { return c == '\t' || c == ',' || c == ' '; }

// (vid_t)atoi(token), token = [b, e): glibc atoi is (int)strtol(s, NULL, 10):
// leading isspace() characters, an optional sign, decimal digits; strtol
// saturates at LONG_MAX / LONG_MIN and the int conversion keeps the low 32
// bits.  A token holds no delimiter, so only \n \v \f \r can lead it.
__device__ uint32_t ref_atoi(const char* __restrict__ t, uint64_t b, uint64_t e) {
  while (b < e) {
    const char c = t[b];
    if (c != '\n' && c != '\v' && c != '\f' && c != '\r') break;
    ++b;
  }
  bool neg = false;
  if (b < e && (t[b] == '+' || t[b] == '-')) {
    neg = t[b] == '-';
    ++b;
  }
  unsigned long long v = 0;
  bool over = false;
  for (; b < e; ++b) {
    const char c = t[b];
    if (c < '0' || c > '9') break;
    if (!over) {
      if (v > (~0ull - 9) / 10) over = true;
      else v = v * 10 + (unsigned long long)(c - '0');
    }
  }
  long long r;
  if (!neg) r = (over || v > 0x7fffffffffffffffull) ? 0x7fffffffffffffffll : (long long)v;
  else r = (over || v > 0x8000000000000000ull) ? (long long)0x8000000000000000ull : (long long)(0ull - v);
  return (uint32_t)(unsigned long long)r;
}

// One thread per line [starts[l], starts[l+1]) of the chunk: the body of
// convert_to_csr's read loop (conversions.hpp:219-241).
__global__ void parse_lines_kernel(const char* __restrict__ t, uint64_t n, const uint32_t* __restrict__ starts,
                                   uint32_t nlines, unsigned long long* __restrict__ edges,
                                   uint8_t* __restrict__ keep, uint32_t* __restrict__ max_vert,
                                   unsigned long long* __restrict__ bad_line) {
  uint32_t mv = 0;
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nlines; l += gridDim.x * blockDim.x) {
    const uint64_t b = starts[l];
    uint64_t e = l + 1 < nlines ? starts[l + 1] : n;
    bool k = false;
    unsigned long long edge = 0;
    if (e - b > kMaxLine) {
      atomicMin(bad_line, (unsigned long long)l);
    } else {
      for (uint64_t z = b; z < e; ++z)  // the C string ends at a NUL byte
        if (t[z] == '\0') {
          e = z;
          break;
        }
      const bool comment = b < e && (t[b] == '#' || t[b] == '%');
      if (!comment) {
        uint64_t t1 = b;
        while (t1 < e && is_delim(t[t1])) ++t1;
        uint64_t e1 = t1;
        while (e1 < e && !is_delim(t[e1])) ++e1;
        uint64_t t2 = e1;
        while (t2 < e && is_delim(t[t2])) ++t2;
        uint64_t e2 = t2;
        while (e2 < e && !is_delim(t[e2])) ++e2;
        if (t1 == e1 || t2 == e2) {
          atomicMin(bad_line, (unsigned long long)l);
        } else {
          const uint32_t from = ref_atoi(t, t1, e1), to = ref_atoi(t, t2, e2);
          if (from != to) {  // self-loops are skipped (conversions.hpp:239)
            k = true;
            edge = ((unsigned long long)from << 32) | to;
            mv = max(mv, max(from, to));
          }
        }
      }
    }
    edges[l] = edge;
    keep[l] = k ? 1 : 0;
  }
  mv = __reduce_max_sync(__activemask(), mv);
  if ((threadIdx.x & 31) == 0 && mv) atomicMax(max_vert, mv);
}

// flag = 1 when some edge's source is below its predecessor's.
__global__ void unsorted_kernel(const unsigned long long* __restrict__ e, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if ((e[i] >> 32) < (e[i - 1] >> 32)) {
      *flag = 1u;
      return;
    }
}

int grid_of(uint64_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t need = (n + 255) / 256, cap = (uint64_t)sms * 16;
  return (int)(need < cap ? (need ? need : 1) : cap);
}

double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

int remove_tree(const std::string& path) {  // rm_dir (conversions.hpp:42-81)
  DIR* d = opendir(path.c_str());
  if (!d) return -1;
  struct dirent* e;
  while ((e = readdir(d)) != nullptr) {
    if (!strcmp(e->d_name, ".") || !strcmp(e->d_name, "..")) continue;
    const std::string sub = path + "/" + e->d_name;
    struct stat st;
    if (lstat(sub.c_str(), &st) != 0) continue;
    if (S_ISDIR(st.st_mode)) remove_tree(sub);
    else unlink(sub.c_str());
  }
  closedir(d);
  return rmdir(path.c_str());
}

// Host threads for file reads and writes: copies between the page cache and
// user memory run at a few GB/s per thread.
unsigned io_threads() {
  const unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1u : std::min(h, 8u);
}

// pread/pwrite of [off, off + bytes) in slices on io_threads() threads; false
// on an I/O error.  `done` (pread only) receives the bytes transferred.
bool parallel_io(int fd, char* p, size_t bytes, uint64_t off, bool write, size_t* done) {
  const unsigned nt = bytes < (8u << 20) ? 1u : io_threads();
  std::vector<size_t> got(nt, 0);
  std::vector<char> bad(nt, 0);
  auto part = [&](unsigned t) {
    const size_t lo = bytes * t / nt, hi = bytes * (t + 1) / nt;
    size_t k = lo;
    while (k < hi) {
      const ssize_t r = write ? pwrite(fd, p + k, hi - k, (off_t)(off + k)) : pread(fd, p + k, hi - k, (off_t)(off + k));
      if (r < 0) {
        bad[t] = 1;
        break;
      }
      if (r == 0) break;  // end of file
      k += (size_t)r;
    }
    got[t] = k - lo;
  };
  if (nt == 1) {
    part(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(part, t);
    for (auto& x : th) x.join();
  }
  size_t total = 0;
  for (unsigned t = 0; t < nt; ++t) {
    if (bad[t]) return false;
    total += got[t];
  }
  if (done) *done = total;
  return total == bytes || !write;
}

bool write_all(const std::string& path, const void* p, size_t bytes) {
  const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) return false;
  const bool ok = bytes == 0 || parallel_io(fd, const_cast<char*>(static_cast<const char*>(p)), bytes, 0, true, nullptr);
  return close(fd) == 0 && ok;
}

// Device and pinned buffers of one conversion.
struct Converter {
  gw_hostbuf host[2];
  gw_devbuf text, starts, nsel, tmp_edges, keep, edges, edges_alt, scalars, temp, rowptr, colidx;
  cudaStream_t st = nullptr;
  ~Converter() {
    for (auto& h : host) h.release();
    for (gw_devbuf* b : {&text, &starts, &nsel, &tmp_edges, &keep, &edges, &edges_alt, &scalars, &temp, &rowptr, &colidx})
      b->release();
    if (st) cudaStreamDestroy(st);
  }
};

struct FileCloser {
  int fd;
  ~FileCloser() {
    if (fd >= 0) close(fd);
  }
};

#define GW_CV(expr, what)                                                                          \
  do {                                                                                             \
    cudaError_t _e = (expr);                                                                       \
    if (_e != cudaSuccess)                                                                         \
      return thread_error(_e == cudaErrorMemoryAllocation ? GW_E_NOMEM : GW_E_CUDA,                \
                          std::string(what) + ": " + cudaGetErrorString(_e));                      \
  } while (0)

// Grows a device buffer to `bytes`, keeping its first `keep` bytes.
cudaError_t grow(gw_devbuf* b, size_t bytes, size_t keep, cudaStream_t st) {
  if (bytes <= b->bytes && b->p) return cudaSuccess;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return e;
  if (keep) e = cudaMemcpyAsync(p, b->p, keep, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (b->p) cudaFree(b->p);
  b->p = p;
  b->bytes = bytes;
  return e;
}

gw_status convert(const char* path, uint64_t blocksize_kb, int32_t device, gw_convert_stats* out) {
  const auto t_start = std::chrono::steady_clock::now();
  gw_convert_stats s{};
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return thread_error(GW_E_IO, std::string("cannot open ") + path + ": " + strerror(errno));
  const FileCloser closer{fd};
  struct stat fst;
  fstat(fd, &fst);
  s.bytes = (uint64_t)fst.st_size;
  size_t chunk = kChunkBytes;
  if (const char* env = getenv("GW_CONVERT_CHUNK_BYTES")) {
    const unsigned long long v = strtoull(env, nullptr, 10);
    if (v >= 4096 && v <= kChunkBytes) chunk = (size_t)v;
  }
  Converter c;
  GW_CV(cudaSetDevice(device), "cudaSetDevice");
  GW_CV(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking), "stream");
  for (auto& h : c.host) GW_CV(h.ensure(chunk + kMaxLine + 1), "pinned text buffer");
  GW_CV(c.text.ensure(chunk + kMaxLine + 1), "text buffer");
  GW_CV(c.starts.ensure((chunk + kMaxLine + 2) * 4), "line starts");  // a line may be one byte
  GW_CV(c.nsel.ensure(16), "counter");
  GW_CV(c.scalars.ensure(32), "scalars");
  uint32_t* d_maxv = c.scalars.as<uint32_t>();
  uint32_t* d_flag = d_maxv + 1;
  unsigned long long* d_bad = reinterpret_cast<unsigned long long*>(c.scalars.as<char>() + 8);
  GW_CV(cudaMemsetAsync(c.scalars.p, 0, 8, c.st), "scalars");
  // line-start select temp storage, sized for the largest chunk
  size_t sel_bytes = 0, flag_bytes = 0;
  GW_CV(cub::DeviceSelect::If(nullptr, sel_bytes, thrust::counting_iterator<uint64_t>(0), c.starts.as<uint32_t>(),
                              c.nsel.as<uint64_t>(), (int64_t)(chunk + kMaxLine + 1), LineStartAt{nullptr}, c.st),
        "select sizing");
  GW_CV(c.temp.ensure(sel_bytes), "select temp");

  uint64_t ne = 0, lines_before = 0;
  size_t carry = 0;  // bytes of an unfinished line at the head of the next buffer
  int cur = 0;
  bool eof = false;
  double ms_read = 0;
  uint64_t file_pos = 0;
  // reads the next piece of the file behind `carry` bytes of buffer b
  auto fill = [&](int b, size_t head, size_t* got) -> bool {
    const auto t0 = std::chrono::steady_clock::now();
    const size_t want = (size_t)std::min<uint64_t>(chunk - head, s.bytes - file_pos);
    size_t have = 0;
    if (want && (!parallel_io(fd, c.host[b].as<char>() + head, want, file_pos, false, &have) || have != want))
      return false;  // an I/O error, or the file shrank while it was read
    file_pos += have;
    if (file_pos >= s.bytes) eof = true;
    *got = head + have;
    ms_read += ms_since(t0);
    return true;
  };
  uint64_t edge_cap = 0;  // edges the device buffer holds
  size_t avail = 0;
  if (!fill(cur, 0, &avail)) return thread_error(GW_E_IO, std::string("read error on ") + path);
  gw_status status = GW_OK;
  while (avail > 0) {
    // whole lines of this buffer; the unfinished tail moves to the next one
    char* hb = c.host[cur].as<char>();
    size_t n = avail;
    if (!eof) {
      const void* nl = memrchr(hb, '\n', avail);
      if (!nl) {
        status = thread_error(GW_E_INVALID, "line " + std::to_string(lines_before + 1) + " is longer than 1023 bytes");
        break;
      }
      n = (size_t)((const char*)nl - hb) + 1;
    }
    carry = avail - n;
    GW_CV(cudaMemcpyAsync(c.text.p, hb, n, cudaMemcpyHostToDevice, c.st), "text copy");
    size_t sb = c.temp.bytes;
    GW_CV(cub::DeviceSelect::If(c.temp.p, sb, thrust::counting_iterator<uint64_t>(0), c.starts.as<uint32_t>(),
                                c.nsel.as<uint64_t>(), (int64_t)n, LineStartAt{c.text.as<char>()}, c.st),
          "line select");
    uint64_t nlines = 0;
    GW_CV(cudaMemcpyAsync(&nlines, c.nsel.p, 8, cudaMemcpyDeviceToHost, c.st), "line count");
    GW_CV(cudaStreamSynchronize(c.st), "sync");
    GW_CV(c.tmp_edges.ensure(nlines * 8 + 8), "edge buffer");
    GW_CV(c.keep.ensure(nlines + 8), "flags");
    if (ne + nlines > edge_cap) {  // grow by half again, or to the file's edge estimate from this round
      const uint64_t estimate = (uint64_t)((double)s.bytes / (double)std::max<size_t>(n, 1) * (double)nlines * 1.05);
      edge_cap = std::max<uint64_t>({ne + nlines, edge_cap + edge_cap / 2, estimate});
      GW_CV(grow(&c.edges, edge_cap * 8 + 8, ne * 8, c.st), "edge buffer");
    }
    const unsigned long long none = kNoLine;
    GW_CV(cudaMemcpyAsync(d_bad, &none, 8, cudaMemcpyHostToDevice, c.st), "bad line");
    if (nlines) {
      parse_lines_kernel<<<grid_of(nlines), 256, 0, c.st>>>(c.text.as<char>(), n, c.starts.as<uint32_t>(),
                                                            (uint32_t)nlines, c.tmp_edges.as<unsigned long long>(),
                                                            c.keep.as<uint8_t>(), d_maxv, d_bad);
      GW_CV(cudaGetLastError(), "parse");
      size_t fb = 0;
      GW_CV(cub::DeviceSelect::Flagged(nullptr, fb, c.tmp_edges.as<unsigned long long>(), c.keep.as<uint8_t>(),
                                       c.edges.as<unsigned long long>() + ne, c.nsel.as<uint64_t>(),
                                       (int64_t)nlines, c.st),
            "compact sizing");
      if (fb > flag_bytes) flag_bytes = fb;
      GW_CV(grow(&c.temp, std::max(flag_bytes, sel_bytes), 0, c.st), "compact temp");
      GW_CV(cub::DeviceSelect::Flagged(c.temp.p, fb, c.tmp_edges.as<unsigned long long>(), c.keep.as<uint8_t>(),
                                       c.edges.as<unsigned long long>() + ne, c.nsel.as<uint64_t>(),
                                       (int64_t)nlines, c.st),
            "compact");
    } else {
      GW_CV(cudaMemsetAsync(c.nsel.p, 0, 8, c.st), "count");
    }
    uint64_t kept = 0;
    unsigned long long bad = kNoLine;
    GW_CV(cudaMemcpyAsync(&kept, c.nsel.p, 8, cudaMemcpyDeviceToHost, c.st), "edge count");
    GW_CV(cudaMemcpyAsync(&bad, d_bad, 8, cudaMemcpyDeviceToHost, c.st), "bad line");
    // read the next piece while the device parses this one
    const int nxt = cur ^ 1;
    if (carry) memcpy(c.host[nxt].as<char>(), hb + n, carry);
    size_t next_avail = carry;
    if (!eof && !fill(nxt, carry, &next_avail)) {
      status = thread_error(GW_E_IO, std::string("read error on ") + path);
      break;
    }
    GW_CV(cudaStreamSynchronize(c.st), "parse");
    if (bad != kNoLine) {
      status = thread_error(GW_E_INVALID, "line " + std::to_string(lines_before + bad + 1) +
                                              " is not '<from> <to>' or is longer than 1023 bytes");
      break;
    }
    ne += kept;
    lines_before += nlines;
    cur = nxt;
    avail = next_avail;
    if (eof && avail == 0) break;
  }
  if (status != GW_OK) return status;
  s.lines = lines_before;
  s.edges = ne;
  s.ms_read = ms_read;

  // ---- group by source, build the CSR ----
  uint32_t max_vert = 0, flag = 0;
  GW_CV(cudaMemcpyAsync(&max_vert, d_maxv, 4, cudaMemcpyDeviceToHost, c.st), "max vertex");
  if (ne > 1) unsorted_kernel<<<grid_of(ne), 256, 0, c.st>>>(c.edges.as<unsigned long long>(), ne, d_flag);
  GW_CV(cudaMemcpyAsync(&flag, d_flag, 4, cudaMemcpyDeviceToHost, c.st), "order flag");
  GW_CV(cudaStreamSynchronize(c.st), "sync");
  const uint64_t nv = (uint64_t)max_vert + 1;
  s.nvertices = (uint32_t)nv;
  s.sorted = flag ? 0u : 1u;
  const unsigned long long* keys = c.edges.as<unsigned long long>();
  if (flag) {  // stable radix sort on the source bits only
    int bits = 1;
    while (bits < 32 && (max_vert >> bits)) ++bits;
    GW_CV(c.edges_alt.ensure(ne * 8), "sort buffer");
    size_t sb = 0;
    GW_CV(cub::DeviceRadixSort::SortKeys(nullptr, sb, c.edges.as<unsigned long long>(),
                                         c.edges_alt.as<unsigned long long>(), (int64_t)ne, 32, 32 + bits, c.st),
          "sort sizing");
    GW_CV(grow(&c.temp, sb, 0, c.st), "sort temp");
    GW_CV(cub::DeviceRadixSort::SortKeys(c.temp.p, sb, c.edges.as<unsigned long long>(),
                                         c.edges_alt.as<unsigned long long>(), (int64_t)ne, 32, 32 + bits, c.st),
          "sort");
    keys = c.edges_alt.as<unsigned long long>();
  }
  GW_CV(c.rowptr.ensure((nv + 1) * 8), "row pointer");
  GW_CV(c.colidx.ensure(ne * 4 + 4), "column array");
  GW_CV(launch_rowptr_from_sorted(keys, ne, (uint32_t)nv, c.rowptr.as<unsigned long long>(), c.colidx.as<uint32_t>(),
                                  c.st),
        "row pointer");
  std::unique_ptr<uint64_t[]> rowptr(new uint64_t[nv + 1]);  // filled by the copy: no zeroing
  GW_CV(cudaMemcpyAsync(rowptr.get(), c.rowptr.p, (nv + 1) * 8, cudaMemcpyDeviceToHost, c.st), "row pointer copy");
  GW_CV(cudaStreamSynchronize(c.st), "sync");
  s.ms_device = ms_since(t_start) - s.ms_read;

  // ---- the reference's files ----
  const auto t_write = std::chrono::steady_clock::now();
  const std::string dir = std::string(path) + "_GraphWalker";
  remove_tree(dir);
  mkdir(dir.c_str(), 0777);
  mkdir((dir + "/graphinfo").c_str(), 0777);
  bool ok = write_all(dir + "/graphinfo/file_0.beg_pos", rowptr.get(), (nv + 1) * 8);
  {  // the column array goes to the file through the two pinned buffers: copy slice k+1 while slice k is written
    const int cf = open((dir + "/graphinfo/file_0.csr").c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    ok = ok && cf >= 0;
    const size_t slice = chunk / 4 * 4;
    cudaEvent_t copied[2];
    for (auto& ev : copied) GW_CV(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    auto issue = [&](uint64_t off, int b) {
      const size_t m = (size_t)std::min<uint64_t>(slice, ne * 4 - off);
      cudaMemcpyAsync(c.host[b].p, c.colidx.as<char>() + off, m, cudaMemcpyDeviceToHost, c.st);
      cudaEventRecord(copied[b], c.st);
    };
    if (ok && ne) issue(0, 0);
    for (uint64_t off = 0, b = 0; ok && off < ne * 4; off += slice, b ^= 1) {
      if (off + slice < ne * 4) issue(off + slice, (int)(b ^ 1));
      ok = cudaEventSynchronize(copied[b]) == cudaSuccess &&
           parallel_io(cf, c.host[b].as<char>(), (size_t)std::min<uint64_t>(slice, ne * 4 - off), off, true, nullptr);
    }
    cudaStreamSynchronize(c.st);  // no copy may be left writing a pinned buffer
    for (auto& ev : copied) cudaEventDestroy(ev);
    if (cf >= 0 && close(cf) != 0) ok = false;
  }
  const std::string nvs = std::to_string(nv) + "\n";
  ok = ok && write_all(dir + "/filesize_1024GB.filerange", ("0\n" + nvs).data(), 2 + nvs.size()) &&
       write_all(dir + "/N.nvertices", nvs.data(), nvs.size());
  if (ok && blocksize_kb) {
    std::vector<uint32_t> blocks(nv + 2);
    const uint32_t nb = gw_compute_blocks(rowptr.get(), (uint32_t)nv, blocksize_kb, blocks.data(),
                                          (uint32_t)blocks.size());
    std::string txt;
    for (uint32_t i = 0; i < nb; ++i) txt += std::to_string(blocks[i]) + "\n";
    ok = write_all(dir + "/blocksize_" + std::to_string(blocksize_kb) + "KB.blockrange", txt.data(), txt.size());
    s.nblocks = nb ? nb - 1 : 0;
  }
  if (!ok) return thread_error(GW_E_IO, "cannot write the preprocessed files under " + dir);
  s.ms_write = ms_since(t_write);
  s.ms_total = ms_since(t_start);
  if (out) *out = s;
  return GW_OK;
}

}  // namespace
}  // namespace gw

extern "C" gw_status gw_convert_edgelist(const char* path, uint64_t blocksize_kb, int32_t device,
                                         gw_convert_stats* stats) {
  if (!path) return gw::thread_error(GW_E_INVALID, "gw_convert_edgelist: NULL path");
  return gw::convert(path, blocksize_kb, device, stats);
}
