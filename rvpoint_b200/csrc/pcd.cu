// PCD input (io/simple_pcd_loader.h:143-291): the step before the voxel grid.
//
// The header is parsed on the host with the reference's rules (tags FIELDS,
// SIZE, TYPE, COUNT, POINTS, WIDTH-if-no-POINTS, DATA; '#' lines skipped;
// COUNT defaults to 1). The payload goes to the device in the form the file
// holds it and is split there:
//   binary             records of all fields back to back: the records are
//                      read in chunks by several threads into pinned buffers
//                      and copied up while the next chunks are read; one
//                      thread per point picks x, y, z from its record (the
//                      AoS -> SoA transpose runs on the GPU);
//   binary_compressed  one LZF block holding each field's column in turn:
//                      decoded on the host (LZF is a sequential byte stream),
//                      then the x, y, z columns are copied up as they are;
//   ascii              one point per line, parsed on the host.
// x, y, z must be 4-byte fields, as in the reference.
#include <stdio.h>
#include <string.h>

#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

namespace rvp {
namespace {

struct PcdHeader {
  std::vector<std::string> fields;
  std::vector<int> sizes, counts;
  std::vector<char> types;
  size_t points = 0;
  std::string data;
};

bool parse_header(std::istream &in, PcdHeader &h) {
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::stringstream ss(line);
    std::string tag;
    ss >> tag;
    if (tag == "FIELDS") {
      h.fields.clear();
      for (std::string f; ss >> f;) h.fields.push_back(f);
    } else if (tag == "SIZE") {
      h.sizes.clear();
      for (int v; ss >> v;) h.sizes.push_back(v);
    } else if (tag == "TYPE") {
      h.types.clear();
      for (char v; ss >> v;) h.types.push_back(v);
    } else if (tag == "COUNT") {
      h.counts.clear();
      for (int v; ss >> v;) h.counts.push_back(v);
    } else if (tag == "POINTS") {
      ss >> h.points;
    } else if (tag == "WIDTH" && h.points == 0) {
      ss >> h.points;
    } else if (tag == "DATA") {
      ss >> h.data;
      break;
    }
  }
  if (h.fields.empty() || h.sizes.size() != h.fields.size() ||
      h.types.size() != h.fields.size())
    return false;
  if (h.counts.empty()) h.counts.assign(h.fields.size(), 1);
  return h.points > 0 && !h.data.empty();
}

int field(const PcdHeader &h, const char *name) {
  for (size_t i = 0; i < h.fields.size(); ++i)
    if (h.fields[i] == name) return (int)i;
  return -1;
}

// LZF: a control byte c < 32 copies c + 1 literal bytes; otherwise a
// back-reference of length (c >> 5) + 2 (7 -> plus the next byte) at
// distance ((c & 31) << 8 | next byte) + 1.
bool lzf_decode(const std::vector<unsigned char> &in, std::vector<unsigned char> &out) {
  size_t ip = 0, op = 0;
  while (ip < in.size()) {
    unsigned c = in[ip++];
    if (c < 32) {
      const size_t len = c + 1;
      if (ip + len > in.size() || op + len > out.size()) return false;
      memcpy(out.data() + op, in.data() + ip, len);
      ip += len;
      op += len;
    } else {
      size_t len = c >> 5;
      if (ip >= in.size()) return false;
      if (len == 7) {
        len += in[ip++];
        if (ip >= in.size()) return false;
      }
      const size_t back = (((size_t)(c & 31)) << 8) + in[ip++] + 1;
      if (back > op || op + len + 2 > out.size()) return false;
      size_t ref = op - back;
      for (size_t k = 0; k < len + 2; ++k) out[op++] = out[ref++];
    }
  }
  return op == out.size();
}

__global__ void k_pcd_records(const unsigned char *raw, size_t n, size_t stride, size_t ox,
                              size_t oy, size_t oz, float *x, float *y, float *z) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const unsigned char *r = raw + i * stride;
    float v[3];
    memcpy(&v[0], r + ox, 4);  // records need not be 4-byte aligned
    memcpy(&v[1], r + oy, 4);
    memcpy(&v[2], r + oz, 4);
    x[i] = v[0];
    y[i] = v[1];
    z[i] = v[2];
  }
}

}  // namespace
}  // namespace rvp

extern "C" rvp_status rvp_pcd_load(rvp_context *ctx, const char *path, int mem, float *x,
                                   float *y, float *z, size_t capacity, size_t *n_points) {
  using namespace rvp;
  if (!ctx || !path || !n_points) return RVP_ERR_INVALID_ARG;
  try {
    *n_points = 0;
    std::ifstream f(path, std::ios::binary);
    RVP_REQUIRE(f.is_open(), std::string("cannot open ") + path);
    PcdHeader h;
    RVP_REQUIRE(parse_header(f, h), "malformed PCD header");
    const int xi = field(h, "x"), yi = field(h, "y"), zi = field(h, "z");
    RVP_REQUIRE(xi >= 0 && yi >= 0 && zi >= 0, "PCD without x/y/z fields");
    RVP_REQUIRE(h.sizes[xi] == 4 && h.sizes[yi] == 4 && h.sizes[zi] == 4,
                "x/y/z fields must be 4 bytes");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    auto put = [&](float *dst, const float *src, size_t cnt) {
      RVP_CUDA_TRY(cudaMemcpyAsync(dst, src, cnt * 4,
                                   mem == RVP_MEM_DEVICE ? cudaMemcpyHostToDevice
                                                         : cudaMemcpyHostToHost,
                                   st));
    };
    if (h.data == "ascii") {
      std::vector<float> hx, hy, hz;
      std::string line;
      std::vector<float> vals(h.fields.size());
      while (std::getline(f, line)) {
        if (line.empty()) continue;
        std::stringstream ss(line);
        for (auto &v : vals) ss >> v;
        if (ss.fail()) continue;
        hx.push_back(vals[xi]);
        hy.push_back(vals[yi]);
        hz.push_back(vals[zi]);
      }
      *n_points = hx.size();
      if (hx.size() > capacity) throw Error{RVP_ERR_CAPACITY, "capacity below the point count"};
      RVP_REQUIRE(x && y && z, "null output");
      if (!hx.empty()) {
        put(x, hx.data(), hx.size());
        put(y, hy.data(), hy.size());
        put(z, hz.data(), hz.size());
      }
      RVP_CUDA_TRY(cudaStreamSynchronize(st));
      return RVP_OK;
    }
    const size_t n = h.points;
    *n_points = n;
    if (n > capacity) throw Error{RVP_ERR_CAPACITY, "capacity below the point count"};
    RVP_REQUIRE(x && y && z, "null output");
    std::vector<size_t> off(h.fields.size());
    size_t stride = 0;
    for (size_t i = 0; i < h.fields.size(); ++i) {
      off[i] = stride;
      stride += (size_t)h.sizes[i] * (size_t)h.counts[i];
    }
    if (h.data == "binary") {
      if (mem == RVP_MEM_DEVICE) {
        // the records go up as they lie in the file: NB threads read NB
        // chunks at a time (pread) into pinned buffers, and each wave's
        // copies overlap the next wave's reads
        const size_t total = stride * n;
        const long long at0 = (long long)f.tellg();
        RVP_REQUIRE(at0 >= 0, "cannot locate the binary PCD payload");
        DevBuf &d = ctx->scratch[29];
        d.reserve(total);
        constexpr size_t CH = (size_t)8 << 20;
        constexpr int NB = 4;
        cudaEvent_t ev[NB] = {};
        struct Events {  // destroyed on every way out
          cudaEvent_t *e;
          ~Events() {
            for (int i = 0; i < NB; ++i)
              if (e[i]) cudaEventDestroy(e[i]);
          }
        } guard_ev{ev};
        for (int i = 0; i < NB; ++i) {
          ctx->pinned[i].reserve(CH);
          RVP_CUDA_TRY(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
        }
        const int fd = open(path, O_RDONLY);
        RVP_REQUIRE(fd >= 0, std::string("cannot open ") + path);
        struct Fd {
          int fd;
          ~Fd() { close(fd); }
        } guard_fd{fd};
        const size_t chunks = (total + CH - 1) / CH;
        for (size_t w = 0; w < chunks; w += NB) {
          const int nw = (int)std::min<size_t>(NB, chunks - w);
          if (w > 0)  // the buffers' previous copies are done
            for (int i = 0; i < nw; ++i) RVP_CUDA_TRY(cudaEventSynchronize(ev[i]));
          std::atomic<bool> short_read{false};
          auto read_chunk = [&](int i) {
            const size_t at = (w + i) * CH, len = std::min(CH, total - at);
            char *dst = static_cast<char *>(ctx->pinned[i].ptr);
            size_t got = 0;
            while (got < len) {
              const ssize_t r = pread(fd, dst + got, len - got, (off_t)(at0 + at + got));
              if (r <= 0) break;
              got += (size_t)r;
            }
            if (got != len) short_read.store(true);
          };
          std::vector<std::thread> th;
          for (int i = 1; i < nw; ++i) th.emplace_back(read_chunk, i);
          read_chunk(0);
          for (auto &t : th) t.join();
          if (short_read.load()) {
            RVP_CUDA_TRY(cudaStreamSynchronize(st));
            throw Error{RVP_ERR_INVALID_ARG, "short binary PCD payload"};
          }
          for (int i = 0; i < nw; ++i) {
            const size_t at = (w + i) * CH, len = std::min(CH, total - at);
            RVP_CUDA_TRY(cudaMemcpyAsync(d.as<unsigned char>() + at, ctx->pinned[i].ptr, len,
                                         cudaMemcpyHostToDevice, st));
            RVP_CUDA_TRY(cudaEventRecord(ev[i], st));
          }
        }
        k_pcd_records<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, st>>>(
            d.as<unsigned char>(), n, stride, off[xi], off[yi], off[zi], x, y, z);
        RVP_LAUNCH_CHECK(ctx);
        RVP_CUDA_TRY(cudaStreamSynchronize(st));
      } else {
        std::vector<unsigned char> raw(stride * n);
        f.read(reinterpret_cast<char *>(raw.data()), (std::streamsize)raw.size());
        RVP_REQUIRE((size_t)f.gcount() == raw.size(), "short binary PCD payload");
        for (size_t i = 0; i < n; ++i) {
          const unsigned char *r = raw.data() + i * stride;
          memcpy(&x[i], r + off[xi], 4);
          memcpy(&y[i], r + off[yi], 4);
          memcpy(&z[i], r + off[zi], 4);
        }
      }
      return RVP_OK;
    }
    RVP_REQUIRE(h.data == "binary_compressed", "unsupported PCD DATA mode " + h.data);
    uint32_t csize = 0, usize = 0;
    f.read(reinterpret_cast<char *>(&csize), 4);
    f.read(reinterpret_cast<char *>(&usize), 4);
    RVP_REQUIRE((bool)f, "missing compressed sizes");
    std::vector<unsigned char> comp(csize), plain(usize);
    f.read(reinterpret_cast<char *>(comp.data()), (std::streamsize)comp.size());
    RVP_REQUIRE((size_t)f.gcount() == comp.size(), "short compressed PCD payload");
    RVP_REQUIRE(lzf_decode(comp, plain), "corrupt LZF payload");
    // columns: each field's values for all points, in field order
    std::vector<size_t> col(h.fields.size());
    size_t cur = 0;
    for (size_t i = 0; i < h.fields.size(); ++i) {
      col[i] = cur;
      cur += (size_t)h.sizes[i] * (size_t)h.counts[i] * n;
    }
    RVP_REQUIRE(cur <= plain.size(), "decompressed PCD payload too small");
    auto column = [&](int fi, float *dst) {
      const size_t es = (size_t)h.sizes[fi] * (size_t)h.counts[fi];
      if (es == 4) {
        put(dst, reinterpret_cast<const float *>(plain.data() + col[fi]), n);
      } else {  // several values per point: the first of each
        std::vector<float> tmp(n);
        for (size_t i = 0; i < n; ++i) memcpy(&tmp[i], plain.data() + col[fi] + i * es, 4);
        put(dst, tmp.data(), n);
        RVP_CUDA_TRY(cudaStreamSynchronize(st));
      }
    };
    column(xi, x);
    column(yi, y);
    column(zi, z);
    RVP_CUDA_TRY(cudaStreamSynchronize(st));
    return RVP_OK;
  } catch (const Error &e) {
    ctx->last_error = e.msg;
    cudaGetLastError();
    return e.status;
  } catch (const std::bad_alloc &) {
    ctx->last_error = "host allocation failed";
    return RVP_ERR_OOM;
  } catch (...) {
    ctx->last_error = "unknown error";
    return RVP_ERR_CUDA;
  }
}
