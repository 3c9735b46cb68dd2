// msgpu_io.cpp -- the on-disk array formats of the reference at the library's
// boundary, with parallel host decoding.
//
// Formats (qc::ScalarArray<QC_2D>::save / load, scalarArray.cpp:330-420,
// 481-569; header parsing ReadArrayHeader, auxiliary.h:10-45, and
// READ_COMMENTS, aol.cpp:508-531; raw data aol::Vector::loadRaw,
// vec.cpp:393-460):
//   "P<t>" magic, comment lines starting with '#', "<numX> <numY>", "<max>",
//   one separator character, then numX*numY values, x fastest, of type
//     P2 unsigned char ASCII, P5 unsigned char binary (big-endian unsigned
//     short when max > 255), P7 float ASCII, P8 float binary, P9 double
//     binary, Pa unsigned short binary, Pb short binary.
//   Compression by file-name suffix (aol::Bzipifstream / Bzipofstream,
//   hasBzipSuffix / hasGzipSuffix / hasZlibSuffix, aol.cpp:318-328): ".bz2",
//   ".q2bz", ".q3bz" are one bzip2 stream, ".gz", ".svgz", ".zz" zlib or gzip.
//   A displacement is one such file per component, the name made from a
//   printf mask with one %d (qc::MultiArray::save / load, multiArray.h:272-306).
//   ".dm3" / ".dm4": Gatan DigitalMicrograph images (loadDM3,
//   scalarArray.cpp:727-730, qc::DM3Reader).
// Decoding runs on a pool of host threads, one file per thread at a time.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/msgpu.h"

// libbzip2's public streaming interface (bzlib.h of bzip2 1.0), declared here
// because the image ships the library without its header.
extern "C" {
typedef struct {
  char* next_in;
  unsigned int avail_in;
  unsigned int total_in_lo32;
  unsigned int total_in_hi32;
  char* next_out;
  unsigned int avail_out;
  unsigned int total_out_lo32;
  unsigned int total_out_hi32;
  void* state;
  void* (*bzalloc)(void*, int, int);
  void (*bzfree)(void*, void*);
  void* opaque;
} bz_stream;
int BZ2_bzCompressInit(bz_stream* strm, int blockSize100k, int verbosity, int workFactor);
int BZ2_bzCompress(bz_stream* strm, int action);
int BZ2_bzCompressEnd(bz_stream* strm);
int BZ2_bzDecompressInit(bz_stream* strm, int verbosity, int small);
int BZ2_bzDecompress(bz_stream* strm);
int BZ2_bzDecompressEnd(bz_stream* strm);
}

namespace {

constexpr int kBzRun = 0, kBzFinish = 2;
constexpr int kBzOk = 0, kBzRunOk = 1, kBzFinishOk = 3, kBzStreamEnd = 4;

thread_local std::string t_err;

int io_fail(int code, const std::string& msg) {
  t_err = msg;
  return code;
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t n = strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}
bool bzip_suffix(const std::string& f) { return ends_with(f, ".bz2") || ends_with(f, ".q2bz") || ends_with(f, ".q3bz"); }
bool zlib_suffix(const std::string& f) { return ends_with(f, ".gz") || ends_with(f, ".svgz") || ends_with(f, ".zz"); }

int read_file(const std::string& path, std::vector<char>& out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return io_fail(MSGPU_ERR_INVALID_ARG, "Could not open \"" + path + "\" for reading.");
  std::vector<char> buf;
  char chunk[1 << 16];
  size_t got;
  while ((got = fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  fclose(f);
  out.swap(buf);
  return MSGPU_OK;
}

// One bzip2 stream (the reference reads up to BZ_STREAM_END and stops).
int bunzip(const std::vector<char>& in, std::vector<char>& out, const std::string& path) {
  bz_stream s;
  memset(&s, 0, sizeof s);
  if (BZ2_bzDecompressInit(&s, 0, 0) != kBzOk) return io_fail(MSGPU_ERR_CUDA, "bzip2: cannot initialise");
  out.assign(std::max<size_t>(in.size() * 4, 1 << 20), 0);
  s.next_in = const_cast<char*>(in.data());
  s.avail_in = (unsigned)in.size();
  size_t pos = 0;
  int rc;
  for (;;) {
    if (pos == out.size()) out.resize(out.size() * 2);
    s.next_out = out.data() + pos;
    s.avail_out = (unsigned)std::min<size_t>(out.size() - pos, 1u << 30);
    const unsigned before = s.avail_out;
    rc = BZ2_bzDecompress(&s);
    pos += before - s.avail_out;
    if (rc == kBzStreamEnd) break;
    if (rc != kBzOk || (s.avail_in == 0 && s.avail_out != 0)) {
      BZ2_bzDecompressEnd(&s);
      return io_fail(MSGPU_ERR_SIZE, "bzip2: corrupt or truncated stream in \"" + path + "\"");
    }
  }
  BZ2_bzDecompressEnd(&s);
  out.resize(pos);
  return MSGPU_OK;
}

int bzip(const std::string& in, std::vector<char>& out) {
  bz_stream s;
  memset(&s, 0, sizeof s);
  if (BZ2_bzCompressInit(&s, 9, 0, 0) != kBzOk) return io_fail(MSGPU_ERR_CUDA, "bzip2: cannot initialise");
  out.assign(in.size() + in.size() / 100 + 600, 0);
  s.next_in = const_cast<char*>(in.data());
  s.avail_in = (unsigned)in.size();
  size_t pos = 0;
  for (;;) {
    if (pos == out.size()) out.resize(out.size() * 2);
    s.next_out = out.data() + pos;
    s.avail_out = (unsigned)(out.size() - pos);
    const unsigned before = s.avail_out;
    const int rc = BZ2_bzCompress(&s, kBzFinish);
    pos += before - s.avail_out;
    if (rc == kBzStreamEnd) break;
    if (rc != kBzFinishOk && rc != kBzRunOk) {
      BZ2_bzCompressEnd(&s);
      return io_fail(MSGPU_ERR_CUDA, "bzip2: compression failed");
    }
  }
  (void)kBzRun;
  BZ2_bzCompressEnd(&s);
  out.resize(pos);
  return MSGPU_OK;
}

int gunzip(const std::vector<char>& in, std::vector<char>& out, const std::string& path) {
  z_stream s;
  memset(&s, 0, sizeof s);
  if (inflateInit2(&s, 15 | 32) != Z_OK) return io_fail(MSGPU_ERR_CUDA, "zlib: cannot initialise");
  out.assign(std::max<size_t>(in.size() * 4, 1 << 20), 0);
  s.next_in = (Bytef*)in.data();
  s.avail_in = (uInt)in.size();
  size_t pos = 0;
  for (;;) {
    if (pos == out.size()) out.resize(out.size() * 2);
    s.next_out = (Bytef*)out.data() + pos;
    s.avail_out = (uInt)(out.size() - pos);
    const uInt before = s.avail_out;
    const int rc = inflate(&s, Z_NO_FLUSH);
    pos += before - s.avail_out;
    if (rc == Z_STREAM_END) break;
    if ((rc != Z_OK && rc != Z_BUF_ERROR) || (s.avail_in == 0 && s.avail_out != 0)) {
      inflateEnd(&s);
      return io_fail(MSGPU_ERR_SIZE, "zlib: corrupt or truncated stream in \"" + path + "\"");
    }
  }
  inflateEnd(&s);
  out.resize(pos);
  return MSGPU_OK;
}

// The file's bytes after decompression chosen by its suffix.
int load_bytes(const std::string& path, std::vector<char>& bytes) {
  std::vector<char> raw;
  int rc = read_file(path, raw);
  if (rc) return rc;
  if (bzip_suffix(path)) return bunzip(raw, bytes, path);
  if (zlib_suffix(path)) return gunzip(raw, bytes, path);
  bytes.swap(raw);
  return MSGPU_OK;
}

struct Cursor {
  const char* p;
  const char* end;
  bool eof() const { return p >= end; }
  int get() { return p < end ? (unsigned char)*p++ : -1; }
  int peek() const { return p < end ? (unsigned char)*p : -1; }
};

// Whitespace, then any lines starting with '#'.
void skip_comments(Cursor& c) {
  while (!c.eof() && (c.peek() == ' ' || c.peek() == '\n' || c.peek() == '\t' || c.peek() == '\r')) c.get();
  while (!c.eof() && c.peek() == '#') {
    while (!c.eof() && c.get() != '\n') {
    }
  }
}

bool read_int(Cursor& c, long long& v) {
  while (!c.eof() && isspace(c.peek())) c.get();
  bool neg = false;
  if (c.peek() == '-' || c.peek() == '+') neg = (c.get() == '-');
  if (c.eof() || !isdigit(c.peek())) return false;
  long long x = 0;
  while (!c.eof() && isdigit(c.peek())) x = x * 10 + (c.get() - '0');
  v = neg ? -x : x;
  return true;
}

struct Header {
  char t;            // type character after 'P'
  long long nx, ny, max;
  size_t data;       // offset of the first value
};

int parse_header(const std::vector<char>& b, Header& h, const std::string& path) {
  Cursor c{b.data(), b.data() + b.size()};
  const int m0 = c.get(), m1 = c.get();
  if (m0 != 'P') return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": not a 2D array file (magic must start with 'P')");
  h.t = (char)m1;
  if (m1 <= 0 || !strchr("25789ab", m1))
    return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": wrong magic number");
  skip_comments(c);
  if (!read_int(c, h.nx)) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": error reading numX");
  skip_comments(c);
  if (!read_int(c, h.ny)) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": error reading numY");
  skip_comments(c);
  if (!read_int(c, h.max)) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": error reading max");
  c.get();  // the one separator character
  if (h.nx <= 0 || h.ny <= 0) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": empty array");
  h.data = (size_t)(c.p - b.data());
  return MSGPU_OK;
}

template <typename T>
int convert_binary(const std::vector<char>& b, size_t off, size_t count, double* out, bool swap16,
                   const std::string& path) {
  if (b.size() < off + count * sizeof(T)) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": truncated data");
  const char* p = b.data() + off;
  for (size_t i = 0; i < count; ++i) {
    T v;
    memcpy(&v, p + i * sizeof(T), sizeof(T));
    if (swap16) {
      unsigned short u;
      memcpy(&u, &v, 2);
      u = (unsigned short)((u >> 8) | (u << 8));
      memcpy(&v, &u, 2);
    }
    out[i] = (double)v;
  }
  return MSGPU_OK;
}

int decode(const std::vector<char>& b, const Header& h, double* out, const std::string& path) {
  const size_t count = (size_t)h.nx * (size_t)h.ny;
  switch (h.t) {
    case '9': return convert_binary<double>(b, h.data, count, out, false, path);
    case '8': return convert_binary<float>(b, h.data, count, out, false, path);
    case '5':
      if (h.max > 255) return convert_binary<unsigned short>(b, h.data, count, out, true, path);
      return convert_binary<unsigned char>(b, h.data, count, out, false, path);
    case 'a': return convert_binary<unsigned short>(b, h.data, count, out, false, path);
    case 'b': return convert_binary<short>(b, h.data, count, out, false, path);
    case '2':
    case '7': {
      std::string text(b.begin() + (long)h.data, b.end());
      const char* s = text.c_str();
      char* e = nullptr;
      for (size_t i = 0; i < count; ++i) {
        errno = 0;
        const double v = strtod(s, &e);
        if (e == s) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": truncated ASCII data");
        if (h.t == '2' && (v < 0 || v > 255))
          return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": illegal ascii number for unsigned char");
        out[i] = v;
        s = e;
      }
      return MSGPU_OK;
    }
    default: return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": wrong magic number");
  }
}

// --- Gatan DigitalMicrograph 3 and 4 -------------------------------------
// The tag tree of DM3Reader (dm3Import.h:16-438): big-endian header
// (version 3 or 4, length, byte order 1 = little-endian values), then tag
// directories (identifier 20) and tags (21): a big-endian name length and
// name (version 4: a 64-bit size follows), tags "%%%%", an info count and the
// info words (32-bit in version 3, 64-bit in version 4, big-endian), then the
// value(s).  The image is the last ImageList.<i>.ImageData: its Data array
// (offset, element type, count) and Dimensions.0/1 (numX, numY).
struct DmImage {
  int num = -1;
  long long offset = -1, count = -1;
  int type = -1, nx = -1, ny = -1, nz = -1;
};

struct DmParser {
  const std::vector<char>& b;
  size_t pos = 0;
  int version = 3;
  std::vector<std::string> tag;
  std::vector<DmImage> images;
  std::string err;
  explicit DmParser(const std::vector<char>& bytes) : b(bytes) {}

  bool need(size_t n) {
    if (pos + n > b.size()) {
      if (err.empty()) err = "truncated DM file";
      return false;
    }
    return true;
  }
  long long be(int bytes) {
    if (!need(bytes)) return 0;
    unsigned long long v = 0;
    for (int i = 0; i < bytes; ++i) v = (v << 8) | (unsigned char)b[pos + i];
    pos += bytes;
    if (bytes == 2) return (int16_t)v;
    if (bytes == 4) return (int32_t)v;
    return (long long)v;
  }
  long long word() { return be(version == 3 ? 4 : 8); }
  static int type_size(int t) {
    switch (t) {
      case 2: case 4: return 2;
      case 3: case 5: case 6: return 4;
      case 7: case 11: case 12: return 8;
      case 8: case 10: return 1;
      default: return 0;
    }
  }
  bool skip_values(int t, long long n) {
    const int sz = type_size(t);
    if (!sz) {
      err = "DM value type " + std::to_string(t) + " not implemented";
      return false;
    }
    if (n < 0 || !need((size_t)(sz * n))) return false;
    pos += (size_t)(sz * n);
    return true;
  }
  uint32_t le32() {
    if (!need(4)) return 0;
    uint32_t v;
    memcpy(&v, &b[pos], 4);
    pos += 4;
    return v;
  }
  bool in_image(size_t depth, const char* leaf) const {
    return !images.empty() && tag.size() == depth && tag[0] == "ImageList" &&
           images.back().num == atoi(tag[1].c_str()) && tag[2] == "ImageData" && tag[3] == leaf;
  }
  bool read_tag() {
    for (int i = 0; i < 4; ++i) {
      if (!need(1)) return false;
      if (b[pos++] != '%') {
        err = "unexpected character in a DM tag";
        return false;
      }
    }
    const long long n = word();
    if (n < 1 || n > (1 << 20)) {
      err = "DM info size must be positive";
      return false;
    }
    std::vector<long long> info((size_t)n);
    for (long long i = 0; i < n; ++i) info[(size_t)i] = word();
    if (!err.empty()) return false;
    if (n == 1) {
      if (in_image(5, "Dimensions") && info[0] == 5) {
        const int dir = atoi(tag[4].c_str());
        const int v = (int)le32();
        if (dir == 0) images.back().nx = v;
        else if (dir == 1) images.back().ny = v;
        else if (dir == 2) images.back().nz = v;
      } else if (!skip_values((int)info[0], 1)) {
        return false;
      }
    } else if (info[0] == 15) {  // group
      if (info[1] != 0 || (long long)info.size() - 3 != 2 * info[2]) {
        err = "inconsistent DM group";
        return false;
      }
      for (long long i = 0; i < info[2]; ++i)
        if (info[(size_t)(3 + 2 * i)] != 0 || !skip_values((int)info[(size_t)(4 + 2 * i)], 1)) {
          if (err.empty()) err = "length of fieldname has to be zero";
          return false;
        }
    } else if (info[0] == 20) {  // array
      if (info[1] == 15) {
        if (info.size() < 5 || info[2] != 0 || (long long)info.size() - 5 != 2 * info[3]) {
          err = "inconsistent DM array of groups";
          return false;
        }
        const long long ng = info[3], cnt = info[(size_t)(4 + 2 * ng)];
        for (long long j = 0; j < cnt; ++j)
          for (long long i = 0; i < ng; ++i)
            if (!skip_values((int)info[(size_t)(5 + 2 * i)], 1)) return false;
      } else {
        if (info.size() < 3) {
          err = "inconsistent DM array";
          return false;
        }
        if (in_image(4, "Data")) {
          images.back().offset = (long long)pos;
          images.back().type = (int)info[1];
          images.back().count = info[2];
        }
        if (!skip_values((int)info[1], info[2])) return false;
      }
    } else {
      err = "DM numberType " + std::to_string(info[0]) + " not implemented";
      return false;
    }
    tag.pop_back();
    return true;
  }
  // Returns the identifier read (0 at the end of a directory), -1 on error.
  int read_entry(int dirnum) {
    if (!need(1)) return -1;
    const int id = (unsigned char)b[pos++];
    if (id == 0) return 0;
    const long long len = be(2);
    if (len < 0 || !need((size_t)len)) {
      if (err.empty()) err = "negative DM tag name length";
      return -1;
    }
    const std::string name(&b[pos], (size_t)len);
    pos += (size_t)len;
    tag.push_back(len > 0 ? name : (dirnum > -1 ? std::to_string(dirnum) : std::string("nameless")));
    if (tag.size() == 3 && tag[0] == "ImageList" && tag[2] == "ImageData") {
      images.emplace_back();
      images.back().num = atoi(tag[1].c_str());
    }
    if (version == 4) be(8);
    if (id == 21) return read_tag() ? id : -1;
    if (id == 20) {
      if (!need(2)) return -1;
      pos += 2;  // sorted, closed
      const long long nt = word();
      for (long long i = 0; i < nt; ++i)
        if (read_entry((int)i) < 0) return -1;
      tag.pop_back();
      return id;
    }
    err = "invalid DM tag identifier " + std::to_string(id);
    return -1;
  }
  bool parse() {
    version = (int)be(4);
    if (version != 3 && version != 4) {
      err = "unexpected DM version " + std::to_string(version) + ", expected 3 or 4";
      return false;
    }
    word();  // file length
    if (be(4) != 1) {
      err = "DM byte order not implemented";
      return false;
    }
    if (!need(2)) return false;
    pos += 2;
    word();  // number of tags of the root directory
    while (pos < b.size()) {
      const int id = read_entry(-1);
      if (id < 0) return false;
      if (id == 0) break;
      tag.clear();
    }
    return err.empty();
  }
};

int read_dm(const std::string& path, const std::vector<char>& b, double* out, long long capacity, int* nx, int* ny,
            int expect_nx, int expect_ny) {
  DmParser d(b);
  if (!d.parse()) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": " + d.err);
  if (d.images.empty()) return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": No data entry found.");
  const DmImage& im = d.images.back();
  if (im.offset < 0 || im.nx <= 0 || im.ny <= 0)
    return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": incomplete image entry");
  if (nx) *nx = im.nx;
  if (ny) *ny = im.ny;
  if (expect_nx > 0 && (im.nx != expect_nx || im.ny != expect_ny))
    return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": size " + std::to_string(im.nx) + "x" + std::to_string(im.ny) +
                                       " differs from " + std::to_string(expect_nx) + "x" + std::to_string(expect_ny));
  if (!out) return MSGPU_OK;
  const size_t count = (size_t)im.nx * im.ny;
  if ((long long)count > capacity)
    return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": image does not fit the buffer");
  switch (im.type) {  // DM3ImageData::getSaveType (dm3Import.h:37-51)
    case 3: return convert_binary<int32_t>(b, (size_t)im.offset, count, out, false, path);
    case 2: return convert_binary<int16_t>(b, (size_t)im.offset, count, out, false, path);
    case 4: return convert_binary<uint16_t>(b, (size_t)im.offset, count, out, false, path);
    case 5: return convert_binary<uint32_t>(b, (size_t)im.offset, count, out, false, path);
    case 6: return convert_binary<float>(b, (size_t)im.offset, count, out, false, path);
    case 10: return convert_binary<unsigned char>(b, (size_t)im.offset, count, out, false, path);
    default:
      return io_fail(MSGPU_ERR_UNSUPPORTED, "\"" + path + "\": Data type " + std::to_string(im.type) +
                                                " not implemented");
  }
}

// expect_nx/expect_ny > 0: the file must have exactly that size.
int read_one(const std::string& path, double* out, long long capacity, int* nx, int* ny, int expect_nx = 0,
             int expect_ny = 0) {
  std::vector<char> b;
  int rc = load_bytes(path, b);
  if (rc) return rc;
  if (ends_with(path, ".dm3") || ends_with(path, ".dm4"))
    return read_dm(path, b, out, capacity, nx, ny, expect_nx, expect_ny);
  Header h;
  if ((rc = parse_header(b, h, path))) return rc;
  if (nx) *nx = (int)h.nx;
  if (ny) *ny = (int)h.ny;
  if (expect_nx > 0 && (h.nx != expect_nx || h.ny != expect_ny))
    return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": size " + std::to_string(h.nx) + "x" + std::to_string(h.ny) +
                                       " differs from " + std::to_string(expect_nx) + "x" + std::to_string(expect_ny));
  if (!out) return MSGPU_OK;
  if (h.nx * h.ny > capacity)
    return io_fail(MSGPU_ERR_SIZE, "\"" + path + "\": " + std::to_string(h.nx) + "x" + std::to_string(h.ny) +
                                       " values do not fit the buffer of " + std::to_string(capacity));
  return decode(b, h, out, path);
}

int write_one(const std::string& path, const double* data, int nx, int ny, int type) {
  if (!data || nx <= 0 || ny <= 0) return io_fail(MSGPU_ERR_INVALID_ARG, "write: empty array or null data");
  if (type != 8 && type != 9) return io_fail(MSGPU_ERR_UNSUPPORTED, "write: type must be 8 (float) or 9 (double)");
  const size_t count = (size_t)nx * ny;
  double mx = data[0];
  for (size_t i = 1; i < count; ++i) mx = std::max(mx, data[i]);
  std::string s = "P" + std::to_string(type) + "\n# written by libmsgpu\n" + std::to_string(nx) + " " +
                  std::to_string(ny) + "\n" + std::to_string((int)mx) + "\n";
  const size_t hdr = s.size();
  if (type == 9) {
    s.resize(hdr + count * sizeof(double));
    memcpy(&s[hdr], data, count * sizeof(double));
  } else {
    s.resize(hdr + count * sizeof(float));
    for (size_t i = 0; i < count; ++i) {
      const float v = (float)data[i];
      memcpy(&s[hdr + i * sizeof(float)], &v, sizeof(float));
    }
  }
  std::vector<char> outb;
  if (bzip_suffix(path)) {
    int rc = bzip(s, outb);
    if (rc) return rc;
  } else if (zlib_suffix(path)) {
    uLongf len = compressBound((uLong)s.size()) + 64;
    outb.resize(len);
    if (compress2((Bytef*)outb.data(), &len, (const Bytef*)s.data(), (uLong)s.size(), 6) != Z_OK)
      return io_fail(MSGPU_ERR_CUDA, "zlib: compression failed");
    outb.resize(len);
  } else {
    outb.assign(s.begin(), s.end());
  }
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return io_fail(MSGPU_ERR_INVALID_ARG, "Cannot open \"" + path + "\" for writing");
  const size_t w = fwrite(outb.data(), 1, outb.size(), f);
  const int cl = fclose(f);
  if (w != outb.size() || cl != 0) return io_fail(MSGPU_ERR_INVALID_ARG, "write to \"" + path + "\" failed");
  return MSGPU_OK;
}

std::string mask_name(const char* mask, int i) {
  char buf[4096];
  snprintf(buf, sizeof buf, mask, i);
  return buf;
}

int check_mask(const char* mask) {
  if (!mask) return io_fail(MSGPU_ERR_INVALID_ARG, "null file-name mask");
  int pct = 0;
  for (const char* p = mask; *p; ++p) pct += (*p == '%');
  if (pct != 1 || !strstr(mask, "%d")) return io_fail(MSGPU_ERR_INVALID_ARG, "the mask needs exactly one %d");
  return MSGPU_OK;
}

}  // namespace

extern "C" {

const char* msgpu_io_last_error(void) { return t_err.c_str(); }

int msgpu_read_array(const char* path, double* out, long long capacity, int* nx, int* ny) {
  if (!path) return io_fail(MSGPU_ERR_INVALID_ARG, "null path");
  return read_one(path, out, capacity, nx, ny);
}

int msgpu_write_array(const char* path, const double* data, int nx, int ny, int type) {
  if (!path) return io_fail(MSGPU_ERR_INVALID_ARG, "null path");
  return write_one(path, data, nx, ny, type);
}

int msgpu_read_arrays(const char* const* paths, int count, int nx, int ny, double* out, int threads) {
  if (!paths || count < 0 || nx <= 0 || ny <= 0 || (!out && count > 0))
    return io_fail(MSGPU_ERR_INVALID_ARG, "read_arrays: invalid arguments");
  const int nt = std::max(1, std::min(threads < 1 ? (int)std::thread::hardware_concurrency() : threads, count));
  std::atomic<int> next(0);
  std::vector<int> codes(count, MSGPU_OK);
  std::vector<std::string> msgs(count);
  auto work = [&]() {
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= count) break;
      int rc = paths[i] ? read_one(paths[i], out + (size_t)i * nx * ny, (long long)nx * ny, nullptr, nullptr, nx, ny)
                        : io_fail(MSGPU_ERR_INVALID_ARG, "null path");
      if (rc) {
        codes[i] = rc;
        msgs[i] = t_err;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  for (int i = 0; i < count; ++i)
    if (codes[i]) return io_fail(codes[i], msgs[i]);
  return MSGPU_OK;
}

struct msgpu_io_task {
  std::vector<std::string> paths;
  std::thread worker;
  int status = MSGPU_OK;
  std::string err;
};

msgpu_io_task* msgpu_read_arrays_start(const char* const* paths, int count, int nx, int ny, double* out,
                                       int threads) {
  if (!paths || count < 0) {
    io_fail(MSGPU_ERR_INVALID_ARG, "read_arrays_start: invalid arguments");
    return nullptr;
  }
  msgpu_io_task* t = new msgpu_io_task;
  for (int i = 0; i < count; ++i) t->paths.emplace_back(paths[i] ? paths[i] : "");
  t->worker = std::thread([t, count, nx, ny, out, threads]() {
    std::vector<const char*> ptrs;
    for (auto& q : t->paths) ptrs.push_back(q.c_str());
    t->status = msgpu_read_arrays(ptrs.data(), count, nx, ny, out, threads);
    if (t->status) t->err = t_err;
  });
  return t;
}

int msgpu_io_wait(msgpu_io_task* task) {
  if (!task) return io_fail(MSGPU_ERR_INVALID_ARG, "io_wait: null task");
  task->worker.join();
  const int rc = task->status;
  if (rc) t_err = task->err;
  delete task;
  return rc;
}

int msgpu_read_displacement(const char* mask, int nx, int ny, double* out) {
  int rc;
  if ((rc = check_mask(mask))) return rc;
  if (!out || nx <= 0 || ny <= 0) return io_fail(MSGPU_ERR_INVALID_ARG, "read_displacement: invalid arguments");
  for (int c = 0; c < 2; ++c) {
    const std::string name = mask_name(mask, c);
    if ((rc = read_one(name, out + (size_t)c * nx * ny, (long long)nx * ny, nullptr, nullptr, nx, ny))) return rc;
  }
  return MSGPU_OK;
}

int msgpu_write_displacement(const char* mask, const double* phi, int nx, int ny) {
  int rc;
  if ((rc = check_mask(mask))) return rc;
  if (!phi) return io_fail(MSGPU_ERR_INVALID_ARG, "write_displacement: null data");
  for (int c = 0; c < 2; ++c)
    if ((rc = write_one(mask_name(mask, c), phi + (size_t)c * nx * ny, nx, ny, 9))) return rc;
  return MSGPU_OK;
}

}  // extern "C"
