// .npy / .npz ingestion for the C ABI: arrays are read in place from a
// read-only mapping of the file (stored members of an .npz included), so a
// job's rows reach evoc_gpu_knn_graph or the server without a host-side
// copy; deflated .npz members are inflated into a buffer the handle owns.
//
// Formats: the NumPy .npy header (magic, version 1-3, a dict literal with
// 'descr', 'fortran_order', 'shape'); .npz = a ZIP archive of .npy members,
// including the ZIP64 fields NumPy writes.  The graph layouts are the
// reference's (load_graph_csr_npz / load_graph_coo_npz,
// src/graph_construction.rs:117-154).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/evoc_gpu.h"

namespace {

struct Handle {
  void* map = nullptr;  // whole-file mapping
  size_t map_len = 0;
  void* owned = nullptr;  // inflated member
};

struct Mapping {
  const uint8_t* p = nullptr;
  size_t len = 0;
  void* base = nullptr;
};

int map_file(const char* path, Mapping* m) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return EVOC_ERR_ARG;
  struct stat st;
  if (fstat(fd, &st) != 0 || st.st_size <= 0) {
    close(fd);
    return EVOC_ERR_ARG;
  }
  void* p = mmap(nullptr, size_t(st.st_size), PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (p == MAP_FAILED) return EVOC_ERR_ARG;
  m->base = p;
  m->p = static_cast<const uint8_t*>(p);
  m->len = size_t(st.st_size);
  return EVOC_OK;
}

uint16_t rd16(const uint8_t* p) { return uint16_t(p[0] | (p[1] << 8)); }
uint32_t rd32(const uint8_t* p) { return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24); }
uint64_t rd64(const uint8_t* p) { return uint64_t(rd32(p)) | (uint64_t(rd32(p + 4)) << 32); }

// The value following `'key':` in the header dict (up to the next top-level comma).
bool dict_value(const std::string& h, const char* key, std::string* out) {
  const std::string k = std::string("'") + key + "'";
  size_t at = h.find(k);
  if (at == std::string::npos) return false;
  at = h.find(':', at + k.size());
  if (at == std::string::npos) return false;
  at++;
  while (at < h.size() && h[at] == ' ') at++;
  size_t end = at;
  int depth = 0;
  for (; end < h.size(); end++) {
    const char c = h[end];
    if (c == '(') depth++;
    if (c == ')') depth--;
    if ((c == ',' || c == '}') && depth == 0) break;
  }
  *out = h.substr(at, end - at);
  return true;
}

int dtype_code(const std::string& descr, int64_t* itemsize) {
  // descr like '<f4'; byte order '<', '|' or '=' (little-endian host)
  if (descr.size() < 5 || descr.front() != '\'' || descr.back() != '\'') return -1;
  const std::string d = descr.substr(1, descr.size() - 2);
  if (d.size() < 3 || d[0] == '>') return -1;
  const std::string t = d.substr(1);
  struct Entry {
    const char* name;
    int code;
    int64_t size;
  };
  static const Entry table[] = {{"f4", EVOC_NPY_F32, 4}, {"f8", EVOC_NPY_F64, 8}, {"i1", EVOC_NPY_I8, 1},
                                {"u1", EVOC_NPY_U8, 1},  {"i4", EVOC_NPY_I32, 4}, {"i8", EVOC_NPY_I64, 8},
                                {"u4", EVOC_NPY_U32, 4}, {"b1", EVOC_NPY_BOOL, 1}};
  for (const auto& e : table)
    if (t == e.name) {
      *itemsize = e.size;
      return e.code;
    }
  return -1;
}

// Parses an .npy image at p (len bytes) into out (data pointer into p).
int parse_npy(const uint8_t* p, size_t len, evoc_npy_array* out) {
  if (len < 10 || std::memcmp(p, "\x93NUMPY", 6) != 0) return EVOC_ERR_ARG;
  const int major = p[6];
  size_t hlen, off;
  if (major == 1) {
    hlen = rd16(p + 8);
    off = 10;
  } else if (major == 2 || major == 3) {
    if (len < 12) return EVOC_ERR_ARG;
    hlen = rd32(p + 8);
    off = 12;
  } else {
    return EVOC_ERR_UNSUPPORTED;
  }
  if (off + hlen > len) return EVOC_ERR_ARG;
  const std::string h(reinterpret_cast<const char*>(p + off), hlen);
  std::string descr, fortran, shape;
  if (!dict_value(h, "descr", &descr) || !dict_value(h, "fortran_order", &fortran) ||
      !dict_value(h, "shape", &shape))
    return EVOC_ERR_ARG;
  int64_t itemsize = 0;
  const int code = dtype_code(descr, &itemsize);
  if (code < 0) return EVOC_ERR_UNSUPPORTED;
  if (shape.size() < 2 || shape.front() != '(' || shape.back() != ')') return EVOC_ERR_ARG;
  int ndim = 0;
  int64_t count = 1;
  const std::string inner = shape.substr(1, shape.size() - 2);
  size_t i = 0;
  while (i < inner.size()) {
    while (i < inner.size() && (inner[i] == ' ' || inner[i] == ',')) i++;
    if (i >= inner.size()) break;
    char* end = nullptr;
    const long long v = std::strtoll(inner.c_str() + i, &end, 10);
    if (end == inner.c_str() + i || v < 0 || ndim >= 8) return EVOC_ERR_ARG;
    out->shape[ndim++] = v;
    // A shape whose element count or byte size overflows 64 bits cannot
    // describe the file: reject it before the size check below can wrap.
    int64_t next = 0;
    if (__builtin_mul_overflow(count, int64_t(v), &next)) return EVOC_ERR_ARG;
    count = next;
    i = size_t(end - inner.c_str());
  }
  int64_t nbytes = 0;
  if (__builtin_mul_overflow(count, itemsize, &nbytes)) return EVOC_ERR_ARG;
  const size_t bytes = size_t(nbytes);
  if (off + hlen > len || bytes > len - (off + hlen)) return EVOC_ERR_ARG;
  out->ndim = ndim;
  out->dtype = code;
  out->fortran_order = fortran.find("True") != std::string::npos ? 1 : 0;
  out->data = p + off + hlen;
  out->nbytes = int64_t(bytes);
  return EVOC_OK;
}

// One member of a ZIP archive: its data bytes (mapped when stored, inflated
// into *owned when deflated).
int zip_member(const Mapping& m, const char* name, const uint8_t** data, size_t* len, void** owned) {
  const uint8_t* p = m.p;
  const size_t n = m.len;
  if (n < 22) return EVOC_ERR_ARG;
  // end of central directory: scan back over a comment of at most 64 KiB
  size_t eocd = SIZE_MAX;
  for (size_t i = n - 22 + 1; i-- > 0 && n - i <= 22 + 65535;)
    if (rd32(p + i) == 0x06054b50u) {
      eocd = i;
      break;
    }
  if (eocd == SIZE_MAX) return EVOC_ERR_ARG;
  uint64_t entries = rd16(p + eocd + 10), cd_off = rd32(p + eocd + 16);
  if (eocd >= 20 && rd32(p + eocd - 20) == 0x07064b50u) {  // ZIP64 end-of-directory locator
    const uint64_t z = rd64(p + eocd - 20 + 8);
    if (z > n || n - z < 56 || rd32(p + z) != 0x06064b50u) return EVOC_ERR_ARG;
    entries = rd64(p + z + 32);
    cd_off = rd64(p + z + 48);
  }
  const std::string want(name), want_npy = want + ".npy";
  uint64_t at = cd_off;
  for (uint64_t e = 0; e < entries; e++) {
    if (at > n || n - at < 46 || rd32(p + at) != 0x02014b50u) return EVOC_ERR_ARG;
    const uint16_t method = rd16(p + at + 10), nlen = rd16(p + at + 28), xlen = rd16(p + at + 30),
                   clen = rd16(p + at + 32);
    uint64_t csize = rd32(p + at + 20), usize = rd32(p + at + 24), loff = rd32(p + at + 42);
    if (at + 46 + nlen + xlen > n) return EVOC_ERR_ARG;
    const std::string nm(reinterpret_cast<const char*>(p + at + 46), nlen);
    // ZIP64 extra field: the 64-bit values of the fields stored as 0xFFFFFFFF, in this order
    const uint64_t x_end = at + 46 + nlen + xlen;  // within the file (checked above)
    for (uint64_t x = at + 46 + nlen; x + 4 <= x_end;) {
      const uint16_t id = rd16(p + x), sz = rd16(p + x + 2);
      if (sz > x_end - (x + 4)) return EVOC_ERR_ARG;  // a field running past the extra region
      if (id == 0x0001) {
        uint64_t y = x + 4;
        if (usize == 0xFFFFFFFFu && y + 8 <= x + 4 + sz) usize = rd64(p + y), y += 8;
        if (csize == 0xFFFFFFFFu && y + 8 <= x + 4 + sz) csize = rd64(p + y), y += 8;
        if (loff == 0xFFFFFFFFu && y + 8 <= x + 4 + sz) loff = rd64(p + y);
      }
      x += 4 + sz;
    }
    if (nm == want || nm == want_npy) {
      // Subtraction-form bounds: loff and csize may be 64-bit ZIP64 values.
      if (loff > n || n - loff < 30 || rd32(p + loff) != 0x04034b50u) return EVOC_ERR_ARG;
      const uint64_t start = loff + 30 + rd16(p + loff + 26) + rd16(p + loff + 28);
      if (start > n || csize > n - start) return EVOC_ERR_ARG;
      if (method == 0) {
        *data = p + start;
        *len = size_t(csize);
        return EVOC_OK;
      }
      if (method != 8) return EVOC_ERR_UNSUPPORTED;
      // zlib counts in 32 bits: deflated members of 4 GiB or more are not read.
      if (csize > 0xFFFFFFFFull || usize > 0xFFFFFFFFull) return EVOC_ERR_UNSUPPORTED;
      void* buf = std::malloc(usize ? size_t(usize) : 1);
      if (!buf) return EVOC_ERR_OOM;
      z_stream zs = {};
      if (inflateInit2(&zs, -MAX_WBITS) != Z_OK) {
        std::free(buf);
        return EVOC_ERR_ARG;
      }
      zs.next_in = const_cast<Bytef*>(p + start);
      zs.avail_in = uInt(csize);
      zs.next_out = static_cast<Bytef*>(buf);
      zs.avail_out = uInt(usize);
      const int rc = inflate(&zs, Z_FINISH);
      inflateEnd(&zs);
      if (rc != Z_STREAM_END || zs.total_out != usize) {
        std::free(buf);
        return EVOC_ERR_ARG;
      }
      *owned = buf;
      *data = static_cast<const uint8_t*>(buf);
      *len = size_t(usize);
      return EVOC_OK;
    }
    at += 46 + nlen + xlen + clen;
  }
  return EVOC_ERR_ARG;  // no such member
}

int open_member(const char* path, const char* name, evoc_npy_array* out) {
  if (!path || !out) return EVOC_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  Mapping m;
  int rc = map_file(path, &m);
  if (rc) return rc;
  const uint8_t* p = m.p;
  size_t len = m.len;
  void* owned = nullptr;
  if (name) {
    rc = zip_member(m, name, &p, &len, &owned);
    if (rc) {
      munmap(m.base, m.len);
      return rc;
    }
  }
  rc = parse_npy(p, len, out);
  if (rc) {
    std::free(owned);
    munmap(m.base, m.len);
    std::memset(out, 0, sizeof(*out));
    return rc;
  }
  Handle* h = new Handle{m.base, m.len, owned};
  out->handle = h;
  return EVOC_OK;
}

void close_member(evoc_npy_array* a) {
  if (!a || !a->handle) return;
  Handle* h = static_cast<Handle*>(a->handle);
  std::free(h->owned);
  if (h->map) munmap(h->map, h->map_len);
  delete h;
  std::memset(a, 0, sizeof(*a));
}

int64_t elems(const evoc_npy_array& a) {
  int64_t c = 1;
  for (int i = 0; i < a.ndim; i++) c *= a.shape[i];
  return c;
}

int64_t as_i64(const evoc_npy_array& a, int64_t i) {
  switch (a.dtype) {
    case EVOC_NPY_I64: return static_cast<const int64_t*>(a.data)[i];
    case EVOC_NPY_I32: return static_cast<const int32_t*>(a.data)[i];
    case EVOC_NPY_U32: return static_cast<const uint32_t*>(a.data)[i];
    default: return INT64_MIN;
  }
}

int graph_read(const char* path, int64_t* n_out, int64_t* nnz_out, int64_t* indptr, int32_t* indices, float* data,
               int64_t cap) {
  if (!path || !n_out || !nnz_out) return EVOC_ERR_ARG;
  evoc_npy_array shape{}, a{}, b{}, w{};
  struct Closer {
    evoc_npy_array* xs[4];
    ~Closer() {
      for (auto* x : xs) close_member(x);
    }
  } closer{{&shape, &a, &b, &w}};
  int rc = open_member(path, "shape", &shape);
  if (rc) return rc;
  if (elems(shape) < 1) return EVOC_ERR_ARG;
  const int64_t n = as_i64(shape, 0);
  const bool csr = open_member(path, "indptr", &a) == EVOC_OK;
  if (!csr && (rc = open_member(path, "rows", &a))) return rc;
  if ((rc = open_member(path, csr ? "indices" : "cols", &b))) return rc;
  if ((rc = open_member(path, "data", &w))) return rc;
  if (w.dtype != EVOC_NPY_F32 || n < 0) return EVOC_ERR_UNSUPPORTED;
  const int64_t nnz = elems(w);
  if (elems(b) != nnz || (csr ? elems(a) != n + 1 : elems(a) != nnz)) return EVOC_ERR_ARG;
  *n_out = n;
  *nnz_out = nnz;
  if (!indptr) return EVOC_OK;  // size query
  if (!indices || !data) return EVOC_ERR_ARG;
  if (cap < nnz) return EVOC_ERR_ARG;
  const float* wv = static_cast<const float*>(w.data);
  if (csr) {
    for (int64_t i = 0; i <= n; i++) indptr[i] = as_i64(a, i);
    if (indptr[0] != 0 || indptr[n] != nnz) return EVOC_ERR_ARG;
    for (int64_t e = 0; e < nnz; e++) {
      const int64_t c = as_i64(b, e);
      if (c < 0 || c >= n) return EVOC_ERR_ARG;
      indices[e] = int32_t(c);
      data[e] = wv[e];
    }
    return EVOC_OK;
  }
  // COO -> CSR with sorted columns; entries with the same (row, column) are summed in file order
  std::vector<int64_t> order(static_cast<size_t>(nnz));
  std::iota(order.begin(), order.end(), 0);
  for (int64_t e = 0; e < nnz; e++) {
    const int64_t r = as_i64(a, e), c = as_i64(b, e);
    if (r < 0 || r >= n || c < 0 || c >= n) return EVOC_ERR_ARG;
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
    const int64_t rx = as_i64(a, x), ry = as_i64(a, y);
    return rx != ry ? rx < ry : as_i64(b, x) < as_i64(b, y);
  });
  std::fill(indptr, indptr + n + 1, int64_t(0));
  int64_t out = 0, prev_r = -1, prev_c = -1;
  for (const int64_t e : order) {
    const int64_t r = as_i64(a, e), c = as_i64(b, e);
    if (r == prev_r && c == prev_c) {
      data[out - 1] += wv[e];
      continue;
    }
    indices[out] = int32_t(c);
    data[out] = wv[e];
    indptr[r + 1]++;
    out++;
    prev_r = r;
    prev_c = c;
  }
  for (int64_t i = 0; i < n; i++) indptr[i + 1] += indptr[i];
  *nnz_out = out;
  return EVOC_OK;
}

}  // namespace

extern "C" {

int evoc_npy_open(const char* path, evoc_npy_array* out) { return open_member(path, nullptr, out); }

int evoc_npz_open(const char* path, const char* name, evoc_npy_array* out) {
  if (!name) return EVOC_ERR_ARG;
  return open_member(path, name, out);
}

void evoc_npy_close(evoc_npy_array* a) { close_member(a); }

int evoc_graph_npz_read(const char* path, int64_t* n, int64_t* nnz, int64_t* indptr, int32_t* indices, float* data,
                        int64_t cap) {
  return graph_read(path, n, nnz, indptr, indices, data, cap);
}

}  // extern "C"
