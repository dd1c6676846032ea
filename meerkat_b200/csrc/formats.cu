// formats.cu -- the reference drivers' text formats (host code).
//
//   graph file    "V E", then E pairs "u v"            (src/BFS.cu:27-36)
//   batch file    "<prefix>.batch.<i>": "n", then n pairs "u v"
//                                                       (src/BFS.cu:76-91)
//
// Tokens are unsigned decimal integers separated by any whitespace.  Unlike
// the reference drivers, which fscanf without checking, a short file, a
// token that is not a number, a number above 32 bits or (graph files) a
// vertex id >= V is an error with the position in the message.  Weights are
// not part of either format: the reference drivers draw them at load time.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mk_internal.h"

namespace mk {
namespace {

struct Text {
  std::vector<char> buf;
  size_t pos = 0;
  size_t line = 1;
};

mk_status load(const char *path, Text &t, const char *what) {
  if (!path) return fail(MK_ERR_INVALID, std::string(what) + ": null path");
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return fail(MK_ERR_INVALID, std::string(what) + ": cannot open " + path + ": " + std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (size < 0) {
    std::fclose(f);
    return fail(MK_ERR_INVALID, std::string(what) + ": cannot size " + path);
  }
  t.buf.resize((size_t)size + 1);
  const size_t got = size ? std::fread(t.buf.data(), 1, (size_t)size, f) : 0;
  std::fclose(f);
  if (got != (size_t)size) return fail(MK_ERR_INVALID, std::string(what) + ": short read of " + path);
  t.buf[(size_t)size] = '\0';
  return MK_OK;
}

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Next unsigned 32-bit token; 0 = ok, 1 = end of text, 2 = bad token.
int next_u32(Text &t, uint32_t &out) {
  const char *b = t.buf.data();
  const size_t n = t.buf.size() - 1;
  while (t.pos < n && is_space(b[t.pos])) {
    if (b[t.pos] == '\n') ++t.line;
    ++t.pos;
  }
  if (t.pos >= n) return 1;
  uint64_t v = 0;
  size_t digits = 0;
  while (t.pos < n && b[t.pos] >= '0' && b[t.pos] <= '9') {
    v = v * 10 + (uint64_t)(b[t.pos] - '0');
    if (v > 0xFFFFFFFFull) return 2;
    ++t.pos;
    ++digits;
  }
  if (digits == 0 || (t.pos < n && !is_space(b[t.pos]))) return 2;
  out = (uint32_t)v;
  return 0;
}

mk_status token(Text &t, uint32_t &out, const char *what, const char *path, const char *field) {
  const int r = next_u32(t, out);
  if (r == 0) return MK_OK;
  return fail(MK_ERR_INVALID, std::string(what) + ": " + path + " line " + std::to_string(t.line) +
                                  (r == 1 ? ": file ends before " : ": not an unsigned 32-bit number: ") +
                                  field);
}

// Parses `count` pairs into h_src / h_dst; ids must be < limit (0 = no limit).
mk_status pairs(Text &t, uint64_t count, uint32_t limit, uint32_t *h_src, uint32_t *h_dst,
                const char *what, const char *path) {
  for (uint64_t i = 0; i < count; ++i) {
    uint32_t u = 0, v = 0;
    bool ok = next_u32(t, u) == 0 && next_u32(t, v) == 0;
    if (!ok || (limit && (u >= limit || v >= limit))) {
      // re-derive the message only on the error path
      const std::string field = "edge " + std::to_string(i) + " of " + std::to_string(count);
      if (ok)
        return fail(MK_ERR_INVALID, std::string(what) + ": " + path + " line " + std::to_string(t.line) +
                                        ": vertex id out of range in " + field);
      return fail(MK_ERR_INVALID, std::string(what) + ": " + path + " line " + std::to_string(t.line) +
                                      ": missing or malformed " + field);
    }
    h_src[i] = u;
    h_dst[i] = v;
  }
  return MK_OK;
}

// Decimal text writer.
struct Out {
  std::FILE *f;
  std::vector<char> buf;
  explicit Out(std::FILE *file) : f(file) { buf.reserve(1 << 20); }
  void num(uint64_t v) {
    char tmp[24];
    int k = 0;
    do {
      tmp[k++] = (char)('0' + v % 10);
      v /= 10;
    } while (v);
    while (k) buf.push_back(tmp[--k]);
  }
  void ch(char c) { buf.push_back(c); }
  bool flush() {
    const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    buf.clear();
    return ok;
  }
};

mk_status write_pairs(const char *path, bool header2, uint64_t a, uint64_t b, uint64_t n,
                      const uint32_t *h_src, const uint32_t *h_dst, const char *what) {
  if (!path || (n && (!h_src || !h_dst))) return fail(MK_ERR_INVALID, std::string(what) + ": null argument");
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return fail(MK_ERR_INVALID, std::string(what) + ": cannot create " + path + ": " + std::strerror(errno));
  Out o(f);
  bool ok = true;
  o.num(a);
  if (header2) {
    o.ch(' ');
    o.num(b);
  }
  o.ch('\n');
  for (uint64_t i = 0; i < n && ok; ++i) {
    o.num(h_src[i]);
    o.ch(' ');
    o.num(h_dst[i]);
    o.ch('\n');
    if (o.buf.size() > (1u << 20) - 32) ok = o.flush();
  }
  ok = ok && o.flush();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(MK_ERR_INVALID, std::string(what) + ": write to " + path + " failed");
  return MK_OK;
}

}  // namespace
}  // namespace mk

using namespace mk;

extern "C" {

mk_status mk_read_edge_list(const char *path, uint32_t *h_num_vertices, uint64_t *h_num_edges,
                            uint32_t *h_src, uint32_t *h_dst) {
  const char *what = "mk_read_edge_list";
  if (!h_num_vertices || !h_num_edges) return fail(MK_ERR_INVALID, std::string(what) + ": null argument");
  Text t;
  MK_CHECK(load(path, t, what));
  uint32_t V = 0, E = 0;
  MK_CHECK(token(t, V, what, path, "the vertex count"));
  MK_CHECK(token(t, E, what, path, "the edge count"));
  *h_num_vertices = V;
  *h_num_edges = E;
  if (!h_src && !h_dst) return MK_OK;  // header query
  if (!h_src || !h_dst) return fail(MK_ERR_INVALID, std::string(what) + ": null edge array");
  return pairs(t, E, V, h_src, h_dst, what, path);
}

mk_status mk_read_batch_file(const char *path, uint64_t *h_num_edges, uint32_t *h_src,
                             uint32_t *h_dst) {
  const char *what = "mk_read_batch_file";
  if (!h_num_edges) return fail(MK_ERR_INVALID, std::string(what) + ": null argument");
  Text t;
  MK_CHECK(load(path, t, what));
  uint32_t n = 0;
  MK_CHECK(token(t, n, what, path, "the edge count"));
  *h_num_edges = n;
  if (!h_src && !h_dst) return MK_OK;
  if (!h_src || !h_dst) return fail(MK_ERR_INVALID, std::string(what) + ": null edge array");
  return pairs(t, n, 0, h_src, h_dst, what, path);
}

mk_status mk_write_edge_list(const char *path, uint32_t num_vertices, uint64_t num_edges,
                             const uint32_t *h_src, const uint32_t *h_dst) {
  if (num_edges > 0xFFFFFFFFull) return fail(MK_ERR_INVALID, "mk_write_edge_list: more than 2^32-1 edges");
  for (uint64_t i = 0; i < num_edges && h_src && h_dst; ++i)
    if (h_src[i] >= num_vertices || h_dst[i] >= num_vertices)
      return fail(MK_ERR_INVALID, "mk_write_edge_list: vertex id out of range at edge " + std::to_string(i));
  return write_pairs(path, true, num_vertices, num_edges, num_edges, h_src, h_dst, "mk_write_edge_list");
}

mk_status mk_write_batch_file(const char *path, uint64_t num_edges, const uint32_t *h_src,
                              const uint32_t *h_dst) {
  if (num_edges > 0xFFFFFFFFull) return fail(MK_ERR_INVALID, "mk_write_batch_file: more than 2^32-1 edges");
  return write_pairs(path, false, num_edges, 0, num_edges, h_src, h_dst, "mk_write_batch_file");
}

}  // extern "C"
