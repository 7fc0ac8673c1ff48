// Configuration files: the reference's reader formats, read straight into
// device-resident links, and its writer format.
//
// Reference: Data::read_data / read_data_convert (data.h:114-173, 248-338),
// file patterns (indexing.h:190-351), MatrixConverter (matrix.h:1104-1119),
// write_data (data.h:175-205).
//
// The payload bytes are read from the file on the host (one read into pinned
// memory), copied to the device once, and one thread per link applies the
// file pattern, the element order, float->double, the big-endian swap of ILDG
// and the optional conversion, writing the structure-of-arrays fields.
//
// ILDG files are LIME containers; the links are the record of type
// "ildg-binary-data". A LIME record is a 144-byte header (big-endian magic
// 0x456789ab, 16-bit version, 16-bit flags, 64-bit payload length, 128-byte
// type string) followed by the payload padded to a multiple of 8 bytes.
#include "../../include/gc_lattice.h"
#include "gc_internal.cuh"
#include "gc_kernels.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>

namespace gc {

int record_error(int code, const std::string &msg);

namespace {

enum FileFormat { kLexicographical = 0, kQcdstag = 1, kIldg = 2 };

__device__ __forceinline__ double read_elem(const unsigned char *p, long long idx,
                                            int single, int swap) {
  if (single) {
    float f;
    memcpy(&f, p + idx * 4, 4);
    return (double)f;
  }
  unsigned long long u;
  memcpy(&u, p + idx * 8, 8);
  if (swap)
    u = __byte_perm((unsigned)(u >> 32), 0, 0x0123) |
        ((unsigned long long)__byte_perm((unsigned)u, 0, 0x0123) << 32);
  return __longlong_as_double((long long)u);
}

template <class Store>
__global__ void file_to_soa_su3(Geom g, const unsigned char *__restrict__ data,
                                int format, int single, int convert, Fields4 U) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4LL * g.V)
    return;
  const int site = (int)(l >> 2), mu = (int)(l & 3);
  long long base;
  if (format == kQcdstag) {
    const int mu1 = (mu == 3) ? 0 : mu + 1; // time direction first
    base = ((long long)site + (long long)mu1 * g.V) * 18;
  } else {
    base = l * 18;
  }
  const int swap = (format == kIldg);
  SU3<double> m;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      m.e[i][j] = {read_elem(data, base + (3 * i + j) * 2, single, swap),
                   read_elem(data, base + (3 * i + j) * 2 + 1, single, swap)};
  if (convert) {
    // A ^ B with B = diag(A_cc / |A_cc|)  (matrix.h:1110-1119)
    SU3<double> B = unit(SU3<double>());
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double n = sqrt(m.e[c][c].re * m.e[c][c].re + m.e[c][c].im * m.e[c][c].im);
      B.e[c][c] = {m.e[c][c].re / n, m.e[c][c].im / n};
    }
    m = mul_ad(m, B);
  }
  Store::template store<double>(U.f[mu], g.V, site, m);
}

template <class Store>
__global__ void file_to_soa_su2(Geom g, const unsigned char *__restrict__ data,
                                int format, int single, int convert, Fields4 U) {
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= 4LL * g.V)
    return;
  const int site = (int)(l >> 2), mu = (int)(l & 3);
  long long base;
  double a[4];
  const int swap = (format == kIldg);
  if (format == kQcdstag) {
    const int mu1 = (mu == 3) ? 0 : mu + 1;
    base = ((long long)site + (long long)mu1 * g.V) * 4;
    // element order a0, a3, a2, a1 (FilePatternQCDSTAG<4, su2>, indexing.h:290-294)
    a[0] = read_elem(data, base, single, swap);
    a[1] = read_elem(data, base + 3, single, swap);
    a[2] = read_elem(data, base + 2, single, swap);
    a[3] = read_elem(data, base + 1, single, swap);
  } else {
    base = l * 4;
    for (int e = 0; e < 4; e++)
      a[e] = read_elem(data, base + e, single, swap);
  }
  SU2<double> m{a[0], a[1], a[2], a[3]};
  if (convert) {
    // A ^ B with B = (a0, 0, 0, a3)/sqrt(a0^2 + a3^2)  (matrix.h:1104-1108)
    const double n = sqrt(m.a0 * m.a0 + m.a3 * m.a3);
    m = mul_ad(m, SU2<double>{m.a0 / n, 0.0, 0.0, m.a3 / n});
  }
  Store::template store<double>(U.f[mu], g.V, site, m);
}

unsigned long long be64(const unsigned char *p) {
  unsigned long long v = 0;
  for (int i = 0; i < 8; i++)
    v = (v << 8) | p[i];
  return v;
}

// Locates the payload of a configuration file. Returns GC_OK and fills
// offset/length (bytes) or an error code with a message.
int locate_payload(const char *path, int format, long long bytes_skip,
                   long long need, long long *offset, std::string &err) {
  struct stat st;
  if (stat(path, &st) != 0) {
    err = std::string("cannot open ") + path;
    return GC_ERR_IO;
  }
  const long long fsize = (long long)st.st_size;
  if (format != kIldg) {
    if (bytes_skip < 0) {
      err = "bytes_skip must be >= 0";
      return GC_ERR_ARG;
    }
    if (fsize < bytes_skip + need) {
      err = std::string(path) + ": file has " + std::to_string(fsize) +
            " bytes, the lattice needs " + std::to_string(bytes_skip + need);
      return GC_ERR_IO;
    }
    *offset = bytes_skip;
    return GC_OK;
  }
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open ") + path;
    return GC_ERR_IO;
  }
  long long pos = 0;
  int rc = GC_ERR_IO;
  err = std::string(path) + ": no ildg-binary-data record";
  while (pos + 144 <= fsize) {
    unsigned char hdr[144];
    if (std::fseek(f, (long)pos, SEEK_SET) != 0 || std::fread(hdr, 1, 144, f) != 144) {
      err = std::string(path) + ": truncated LIME header";
      break;
    }
    const unsigned magic = (unsigned)hdr[0] << 24 | (unsigned)hdr[1] << 16 |
                           (unsigned)hdr[2] << 8 | hdr[3];
    if (magic != 0x456789abu) {
      err = std::string(path) + ": not a LIME file (bad record magic)";
      break;
    }
    const long long len = (long long)be64(hdr + 8);
    char type[129];
    std::memcpy(type, hdr + 16, 128);
    type[128] = 0;
    const long long data = pos + 144;
    if (len < 0 || data + len > fsize) {
      err = std::string(path) + ": truncated LIME record";
      break;
    }
    if (std::strcmp(type, "ildg-binary-data") == 0) {
      if (len < need) {
        err = std::string(path) + ": ildg-binary-data has " + std::to_string(len) +
              " bytes, the lattice needs " + std::to_string(need);
        break;
      }
      *offset = data;
      rc = GC_OK;
      break;
    }
    pos = data + ((len + 7) / 8) * 8;
  }
  std::fclose(f);
  return rc;
}

int parse_format(const char *format) {
  if (!format)
    return -1;
  if (!std::strcmp(format, "lexicographical"))
    return kLexicographical;
  if (!std::strcmp(format, "qcdstag"))
    return kQcdstag;
  if (!std::strcmp(format, "ildg"))
    return kIldg;
  return -1;
}

int parse_precision(const char *precision, int format) {
  if (format == kIldg)
    return 0; // ILDG payloads are read as doubles (data.h:159-166)
  if (precision && !std::strcmp(precision, "float"))
    return 1;
  if (precision && !std::strcmp(precision, "double"))
    return 0;
  return -1;
}

} // namespace

int probe_config(const int dims[4], int nc, const char *path, const char *format,
                 long long bytes_skip, const char *precision, long long *offset,
                 long long *length, std::string &err) {
  const int fmt = parse_format(format);
  if (fmt < 0) {
    err = "format must be lexicographical, qcdstag or ildg";
    return GC_ERR_ARG;
  }
  const int single = parse_precision(precision, fmt);
  if (single < 0) {
    err = "precision must be float or double";
    return GC_ERR_ARG;
  }
  long long V = 1;
  for (int d = 0; d < 4; d++)
    V *= dims[d];
  const long long need = 4 * V * (nc == 3 ? 18 : 4) * (single ? 4 : 8);
  *length = need;
  return locate_payload(path, fmt, bytes_skip, need, offset, err);
}

int launch_file_to_soa(const Geom &g, int nc, int prec, const char *format,
                       const char *precision, int convert, const unsigned char *data,
                       const Fields4 &U, cudaStream_t s) {
  const int fmt = parse_format(format);
  const int single = parse_precision(precision, fmt);
  const long long n = 4LL * g.V;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (nc == 3) {
    if (prec == GC_PREC_FP64)
      file_to_soa_su3<StoreF64SU3><<<grid, 256, 0, s>>>(g, data, fmt, single, convert, U);
    else
      file_to_soa_su3<StoreF32SU3><<<grid, 256, 0, s>>>(g, data, fmt, single, convert, U);
  } else {
    if (prec == GC_PREC_FP64)
      file_to_soa_su2<StoreF64SU2><<<grid, 256, 0, s>>>(g, data, fmt, single, convert, U);
    else
      file_to_soa_su2<StoreF32SU2><<<grid, 256, 0, s>>>(g, data, fmt, single, convert, U);
  }
  return launch_check("file_to_soa");
}

} // namespace gc

extern "C" int gc_probe_config(const int dims[4], int nc, const char *path,
                               const char *format, long long bytes_skip,
                               const char *precision, long long *offset,
                               long long *length) {
  if (!dims || !path || !offset || !length)
    return gc::record_error(GC_ERR_ARG, "gc_probe_config: null argument");
  if (nc != 2 && nc != 3)
    return gc::record_error(GC_ERR_ARG, "gc_probe_config: nc must be 2 or 3");
  for (int d = 0; d < 4; d++)
    if (dims[d] < 2)
      return gc::record_error(GC_ERR_ARG, "gc_probe_config: every extent must be >= 2");
  std::string err;
  int rc = gc::probe_config(dims, nc, path, format, bytes_skip, precision, offset, length, err);
  if (rc)
    return gc::record_error(rc, "gc_probe_config: " + err);
  return GC_OK;
}
