// io.cpp — host-side formats around the solve (include/mmp.h, "results and files"):
// the MEX front end's dense coupling input, the text |phi| dump of the reference's
// driver and the MAT-file struct the MEX front end saves. Plain C++; no device code.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mmp.h"

namespace {

// ---- MATLAB Level-5 MAT-file writer (the published MAT-File Format: a 128-byte
// header, then tagged data elements padded to 8 bytes; arrays are miMATRIX elements
// holding array flags, dimensions, a name and the column-major data).
enum : uint32_t { miINT8 = 1, miINT32 = 5, miUINT32 = 6, miDOUBLE = 9, miMATRIX = 14 };
enum : uint32_t { mxSTRUCT_CLASS = 2, mxDOUBLE_CLASS = 6 };
constexpr uint32_t kComplexFlag = 0x0800;

struct Buf {
  std::vector<unsigned char> b;
  void raw(const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    b.insert(b.end(), c, c + n);
  }
  void u32(uint32_t v) { raw(&v, 4); }
  void pad8() { b.resize((b.size() + 7) & ~(size_t)7, 0); }
  // one tagged element: tag, data, padding
  void element(uint32_t type, const void* data, size_t n) {
    u32(type);
    u32((uint32_t)n);
    raw(data, n);
    pad8();
  }
};

void array_header(Buf& o, uint32_t cls, bool complex, const std::vector<int32_t>& dims, const char* name) {
  const uint32_t flags[2] = {cls | (complex ? kComplexFlag : 0u), 0u};
  o.element(miUINT32, flags, sizeof(flags));
  o.element(miINT32, dims.data(), dims.size() * sizeof(int32_t));
  o.element(miINT8, name, std::strlen(name));
}

// wrap the sub-elements in `body` as one miMATRIX element
void matrix(Buf& o, const Buf& body) {
  o.u32(miMATRIX);
  o.u32((uint32_t)body.b.size());
  o.raw(body.b.data(), body.b.size());
}

void scalar_field(Buf& o, double v) {
  Buf m;
  array_header(m, mxDOUBLE_CLASS, false, {1, 1}, "");
  m.element(miDOUBLE, &v, sizeof(v));
  matrix(o, m);
}

}  // namespace

namespace mmp_detail {
int set_error(int code, const std::string& msg);  // solver.cu: the text mmp_last_error returns
}

namespace {
int io_fail(int code, const std::string& msg) { return mmp_detail::set_error(code, msg); }
}  // namespace

extern "C" {

int mmp_coupling_from_dense(uint32_t M, const double* q, mmp_nz* out, uint32_t cap, uint32_t* n) {
  if (!q || !n || M == 0) return io_fail(MMP_EINVAL, "bad dense coupling arguments");
  // MATLAB order, p fastest, then k, l, m; zeros are skipped (matlab/mm_propagation.cpp:186-209)
  uint32_t cnt = 0;
  const size_t total = (size_t)M * M * M * M;
  for (size_t idx = 0; idx < total; ++idx) {
    const double v = q[idx];
    if (v == 0.0) continue;
    if (out && cnt < cap) {
      size_t r = idx;
      out[cnt].p = (uint32_t)(r % M); r /= M;
      out[cnt].k = (uint32_t)(r % M); r /= M;
      out[cnt].l = (uint32_t)(r % M); r /= M;
      out[cnt].m = (uint32_t)r;
      out[cnt].value = v;
    }
    ++cnt;
  }
  *n = cnt;
  return MMP_OK;
}

int mmp_write_abs_text(const char* path, uint32_t M, uint32_t nt, const double* phi0, const double* phi) {
  if (!path || !phi || M == 0 || nt == 0) return io_fail(MMP_EINVAL, "bad text dump arguments");
  FILE* f = std::fopen(path, "w");
  if (!f) return io_fail(MMP_EINVAL, std::string("cannot open ") + path);
  // one line per sample: |phi0_p[i]| for every mode, then |phi_p[i]| (simulations/main.cpp:101-103),
  // numbers in the default iostream format (%g, 6 significant digits)
  std::string line;
  char num[64];
  for (uint32_t i = 0; i < nt; ++i) {
    line.clear();
    for (int part = 0; part < 2; ++part) {
      const double* a = part == 0 ? phi0 : phi;
      if (!a) continue;
      for (uint32_t p = 0; p < M; ++p) {
        const double* z = a + 2 * ((size_t)p * nt + i);
        std::snprintf(num, sizeof(num), "%g", std::hypot(z[0], z[1]));
        if (!line.empty()) line += " ; ";
        line += num;
      }
    }
    line += '\n';
    if (std::fwrite(line.data(), 1, line.size(), f) != line.size()) {
      std::fclose(f);
      return io_fail(MMP_EINVAL, std::string("write failed: ") + path);
    }
  }
  return std::fclose(f) == 0 ? MMP_OK : io_fail(MMP_EINVAL, std::string("close failed: ") + path);
}

int mmp_write_mat(const char* path, const char* name, double Z, uint32_t M, uint32_t nt, const double* phi,
                  double cpu_time) {
  if (!path || !phi || M == 0 || nt == 0) return io_fail(MMP_EINVAL, "bad MAT-file arguments");
  if (!name || !*name) name = "output";
  if (std::strlen(name) > 63) return io_fail(MMP_EINVAL, "variable name longer than 63 characters");
  Buf file;
  char text[116];
  std::memset(text, ' ', sizeof(text));
  const char* head = "MATLAB 5.0 MAT-file, written by libmmp_b200";
  std::memcpy(text, head, std::strlen(head));
  file.raw(text, sizeof(text));
  const unsigned char subsys[8] = {0};
  file.raw(subsys, 8);
  const uint16_t version = 0x0100;
  file.raw(&version, 2);
  file.raw("IM", 2);  // endian indicator as written by a little-endian machine

  // struct `name` with fields Z, fields, cpu_time (matlab/mm_propagation.cpp:280-311)
  Buf st;
  array_header(st, mxSTRUCT_CLASS, false, {1, 1}, name);
  const int32_t name_len = 32;  // field-name slot length, including the terminating NUL
  st.u32((4u << 16) | miINT32);  // small data element: 4 bytes of miINT32
  st.raw(&name_len, 4);
  const char* names[3] = {"Z", "fields", "cpu_time"};
  std::vector<char> nbuf(3 * name_len, 0);
  for (int k = 0; k < 3; ++k) std::memcpy(&nbuf[k * name_len], names[k], std::strlen(names[k]));
  st.element(miINT8, nbuf.data(), nbuf.size());
  scalar_field(st, Z);
  {
    Buf m;
    array_header(m, mxDOUBLE_CLASS, true, {(int32_t)M, (int32_t)nt}, "");
    // column-major M x NT: element (p, i) at p + M * i; real part, then imaginary part
    std::vector<double> re((size_t)M * nt), im((size_t)M * nt);
    for (uint32_t p = 0; p < M; ++p)
      for (uint32_t i = 0; i < nt; ++i) {
        re[p + (size_t)M * i] = phi[2 * ((size_t)p * nt + i)];
        im[p + (size_t)M * i] = phi[2 * ((size_t)p * nt + i) + 1];
      }
    m.element(miDOUBLE, re.data(), re.size() * sizeof(double));
    m.element(miDOUBLE, im.data(), im.size() * sizeof(double));
    matrix(st, m);
  }
  scalar_field(st, cpu_time);
  matrix(file, st);

  FILE* f = std::fopen(path, "wb");
  if (!f) return io_fail(MMP_EINVAL, std::string("cannot open ") + path);
  const size_t w = std::fwrite(file.b.data(), 1, file.b.size(), f);
  const int c = std::fclose(f);
  if (w != file.b.size() || c != 0) return io_fail(MMP_EINVAL, std::string("write failed: ") + path);
  return MMP_OK;
}

}  // extern "C"
