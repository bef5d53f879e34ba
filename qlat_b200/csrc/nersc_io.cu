// nersc_io.cu -- NERSC gauge-configuration files, as the reference writes and
// reads them (save_gauge_field / load_gauge_field, qcd.h:66-250):
//   - an ASCII header from "BEGIN_HEADER\n" to "END_HEADER\n" (dimensions,
//     average link trace and plaquette, a simple checksum and a CRC-32 of the
//     data, creator, date, ensemble, beta, sequence number, byte order);
//   - the links as IEEE doubles, sites in the reference order (x fastest), 4
//     links per site, each link its first two rows (6 complex numbers,
//     "4D_SU3_GAUGE") or all three ("4D_SU3_GAUGE_3x3" on reading), big-endian
//     ("IEEE64BIG") unless the header says "IEEE64LITTLE".
// The simple checksum is the sum of the data's 32-bit words in host byte
// order (field_simple_checksum, field-io.h:11-25); CRC32HASH is the CRC-32
// (reflected polynomial 0xEDB88320, the zlib / IEEE 802.3 one) of the data as
// stored in the file (field_crc32, field-io.h:84-88).  Reading checks both and
// reports mismatches instead of failing, like the reference's warnings.
//
// The format code is host-only and needs no GPU; the field-level entry points
// move the links through the GPU (download, plaquette; upload, unitarize).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <string>
#include <vector>

#include "../../include/qlat_b200.h"

namespace qgb
{
void set_last_error(const std::string& msg);
}

namespace
{

int nfail(int code, const std::string& m)
{
  qgb::set_last_error(m);
  return code;
}

// ---- CRC-32 (table-driven, reflected polynomial 0xEDB88320) -----------------

struct Crc32Table {
  uint32_t t[256];
  Crc32Table()
  {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1);
      t[i] = c;
    }
  }
};

uint32_t crc32_update(uint32_t crc, const uint8_t* p, size_t n)
{
  static const Crc32Table tab;
  crc = ~crc;
  for (size_t i = 0; i < n; ++i) crc = tab.t[(crc ^ p[i]) & 0xffu] ^ (crc >> 8);
  return ~crc;
}

uint32_t simple_checksum(const std::vector<double>& d)
{
  uint32_t s = 0;
  const uint8_t* p = (const uint8_t*)d.data();
  for (size_t i = 0; i < d.size() * 2; ++i) {
    uint32_t w;
    memcpy(&w, p + 4 * i, 4);
    s += w;
  }
  return s;
}

void swap8(std::vector<double>& d)
{
  uint8_t* p = (uint8_t*)d.data();
  for (size_t i = 0; i < d.size(); ++i) {
    uint8_t* q = p + 8 * i;
    for (int k = 0; k < 4; ++k) {
      const uint8_t t = q[k];
      q[k] = q[7 - k];
      q[7 - k] = t;
    }
  }
}

bool host_is_little_endian()
{
  const uint32_t one = 1;
  uint8_t b;
  memcpy(&b, &one, 1);
  return b == 1;
}

std::string fmt(const char* f, double v)
{
  char buf[64];
  snprintf(buf, sizeof(buf), f, v);
  return buf;
}

std::string make_header(const int32_t ts[4], double plaq, double trace, uint32_t simple, uint32_t crc,
                        const std::string& creator, const std::string& date, const std::string& ensemble_id,
                        const std::string& ensemble_label, double beta, int64_t seq)
{
  // make_gauge_field_header, qcd.h:66-92 (the date line carries its own newline, as ctime's does)
  std::string h = "BEGIN_HEADER\nHDR_VERSION = 1.0\nDATATYPE = 4D_SU3_GAUGE\n";
  for (int m = 0; m < 4; ++m) h += "DIMENSION_" + std::to_string(m + 1) + " = " + std::to_string(ts[m]) + "\n";
  h += fmt("LINK_TRACE = %.12f\n", trace);
  h += fmt("PLAQUETTE = %.12f\n", plaq);
  char buf[64];
  snprintf(buf, sizeof(buf), "CHECKSUM = %08x\n", simple);
  h += buf;
  snprintf(buf, sizeof(buf), "CRC32HASH = %08x\n", crc);
  h += buf;
  h += "CREATOR = " + creator + "\n";
  h += "ARCHIVE_DATE = " + date;
  h += "ENSEMBLE_ID = " + ensemble_id + "\n";
  h += "ENSEMBLE_LABEL = " + ensemble_label + "\n";
  h += fmt("BETA = %.12f\n", beta);
  snprintf(buf, sizeof(buf), "SEQUENCE_NUMBER = %lld\n", (long long)seq);
  h += buf;
  h += "FLOATING_POINT = IEEE64BIG\nEND_HEADER\n";
  return h;
}

struct Header {
  int32_t ts[4] = {0, 0, 0, 0};
  double plaq = 1.0, trace = 0.0;
  uint32_t simple = 0, crc = 0;
  std::string datatype, floating_point;
};

std::string prop(const std::vector<std::string>& lines, const std::string& key)
{
  for (const std::string& l : lines)
    if (l.compare(0, key.size(), key) == 0) {
      std::string v = l.substr(key.size());
      while (!v.empty() && (v.back() == '\n' || v.back() == '\r')) v.pop_back();
      return v;
    }
  return "";
}

// read_gauge_field_header, qcd.h:94-144
int read_header(const char* path, Header& h)
{
  FILE* f = fopen(path, "rb");
  if (!f) return nfail(QGB_ERR_IO, std::string("cannot open '") + path + "'");
  std::vector<std::string> lines;
  char buf[4096];
  bool ok = fgets(buf, sizeof(buf), f) && std::string(buf) == "BEGIN_HEADER\n";
  while (ok && fgets(buf, sizeof(buf), f)) {
    lines.push_back(buf);
    if (lines.back() == "END_HEADER\n") break;
  }
  fclose(f);
  if (!ok || lines.empty() || lines.back() != "END_HEADER\n")
    return nfail(QGB_ERR_IO, std::string("'") + path + "' is not a NERSC gauge file (no BEGIN_HEADER / END_HEADER)");
  for (int m = 0; m < 4; ++m) h.ts[m] = atoi(prop(lines, "DIMENSION_" + std::to_string(m + 1) + " = ").c_str());
  h.trace = atof(prop(lines, "LINK_TRACE = ").c_str());
  h.plaq = atof(prop(lines, "PLAQUETTE = ").c_str());
  std::string s = prop(lines, "CHECKSUM = ");
  h.simple = s.empty() ? 0u : (uint32_t)strtoul(s.c_str(), nullptr, 16);
  s = prop(lines, "CRC32HASH = ");
  h.crc = s.empty() ? 0u : (uint32_t)strtoul(s.c_str(), nullptr, 16);
  h.datatype = prop(lines, "DATATYPE = ");
  h.floating_point = prop(lines, "FLOATING_POINT = ");
  return QGB_OK;
}

std::string now_ctime()
{
  const time_t now = time(nullptr);
  char buf[64];
  ctime_r(&now, buf);  // "Www Mmm dd hh:mm:ss yyyy\n"
  return buf;
}

long volume_of(const int32_t ts[4]) { return (long)ts[0] * ts[1] * ts[2] * ts[3]; }

// Average link trace: per site sum_m Re tr U_m / 3, divided by 4, summed over
// sites in order, divided by V (gf_avg_link_trace, qcd.cpp:203-226).
double link_trace_of(const double* links, long V)
{
  double sum = 0.0;
  for (long s = 0; s < V; ++s) {
    double t = 0.0;
    for (int m = 0; m < 4; ++m) {
      const double* u = links + (s * 4 + m) * 18;
      t += (u[0] + u[8] + u[16]) / 3.0;
    }
    sum += t / 4.0;
  }
  return sum / (double)V;
}

}  // namespace

extern "C" {

int qgb_nersc_write_host(const char* path, const double* links, const int32_t total_site[4], double plaq,
                         double link_trace, const char* ensemble_id, const char* ensemble_label, const char* creator,
                         const char* date, double beta, int64_t sequence_num, int64_t* file_size)
{
  if (!path || !links || !total_site) return nfail(QGB_ERR_INVALID_ARG, "qgb_nersc_write_host: null argument");
  for (int m = 0; m < 4; ++m)
    if (total_site[m] < 1) return nfail(QGB_ERR_BAD_GEOMETRY, "qgb_nersc_write_host: bad lattice extent");
  const long V = volume_of(total_site);
  // save_gauge_field, qcd.h:146-181: rows 0 and 1 of each link
  std::vector<double> d((size_t)V * 4 * 12);
  for (long s = 0; s < V; ++s)
    for (int m = 0; m < 4; ++m) memcpy(&d[(s * 4 + m) * 12], links + (s * 4 + m) * 18, 12 * sizeof(double));
  const uint32_t simple = simple_checksum(d);  // before the byte-order change
  if (host_is_little_endian()) swap8(d);
  const uint32_t crc = crc32_update(0u, (const uint8_t*)d.data(), d.size() * sizeof(double));
  const std::string header =
      make_header(total_site, plaq, link_trace, simple, crc, creator ? creator : "Qlat", date ? date : now_ctime(),
                  ensemble_id ? ensemble_id : "42", ensemble_label ? ensemble_label : "default-ensemble", beta,
                  sequence_num);
  const std::string partial = std::string(path) + ".partial";
  FILE* f = fopen(partial.c_str(), "wb");
  if (!f) return nfail(QGB_ERR_IO, "qgb_nersc_write_host: cannot create '" + partial + "'");
  bool ok = fwrite(header.data(), 1, header.size(), f) == header.size();
  ok = ok && fwrite(d.data(), sizeof(double), d.size(), f) == d.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) return nfail(QGB_ERR_IO, "qgb_nersc_write_host: write to '" + partial + "' failed");
  if (rename(partial.c_str(), path) != 0) return nfail(QGB_ERR_IO, std::string("qgb_nersc_write_host: rename to '") + path + "' failed");
  if (file_size) *file_size = (int64_t)(d.size() * sizeof(double));
  return QGB_OK;
}

int qgb_nersc_read_header(const char* path, int32_t total_site[4], int32_t* n_rows, int32_t* big_endian, double* plaq,
                          double* link_trace, uint32_t* simple_checksum_out, uint32_t* crc32_out)
{
  if (!path) return nfail(QGB_ERR_INVALID_ARG, "qgb_nersc_read_header: null path");
  Header h;
  const int rc = read_header(path, h);
  if (rc != QGB_OK) return rc;
  if (total_site)
    for (int m = 0; m < 4; ++m) total_site[m] = h.ts[m];
  if (n_rows) *n_rows = h.datatype == "4D_SU3_GAUGE" ? 2 : (h.datatype == "4D_SU3_GAUGE_3x3" ? 3 : 0);
  if (big_endian) *big_endian = h.floating_point == "IEEE64BIG" ? 1 : (h.floating_point == "IEEE64LITTLE" ? 0 : -1);
  if (plaq) *plaq = h.plaq;
  if (link_trace) *link_trace = h.trace;
  if (simple_checksum_out) *simple_checksum_out = h.simple;
  if (crc32_out) *crc32_out = h.crc;
  return QGB_OK;
}

int qgb_nersc_read_host(const char* path, double* links, const int32_t total_site[4], int32_t* checks,
                        int64_t* file_size)
{
  if (!path || !links || !total_site) return nfail(QGB_ERR_INVALID_ARG, "qgb_nersc_read_host: null argument");
  Header h;
  int rc = read_header(path, h);
  if (rc != QGB_OK) return rc;
  for (int m = 0; m < 4; ++m)
    if (h.ts[m] != total_site[m])
      return nfail(QGB_ERR_MISMATCH, std::string("qgb_nersc_read_host: '") + path + "' has another lattice size");
  // load_gauge_field, qcd.h:183-250
  const int rows = h.datatype == "4D_SU3_GAUGE" ? 2 : (h.datatype == "4D_SU3_GAUGE_3x3" ? 3 : 0);
  if (rows == 0) return nfail(QGB_ERR_IO, "qgb_nersc_read_host: unknown DATATYPE '" + h.datatype + "'");
  const bool big = h.floating_point == "IEEE64BIG";
  if (!big && h.floating_point != "IEEE64LITTLE")
    return nfail(QGB_ERR_IO, "qgb_nersc_read_host: unknown FLOATING_POINT '" + h.floating_point + "'");
  const long V = volume_of(total_site);
  const int per_link = 6 * rows;  // doubles
  std::vector<double> d((size_t)V * 4 * per_link);
  FILE* f = fopen(path, "rb");
  if (!f) return nfail(QGB_ERR_IO, std::string("qgb_nersc_read_host: cannot open '") + path + "'");
  // the data are the last bytes of the file, whatever the header's length
  const long nbytes = (long)(d.size() * sizeof(double));
  bool ok = fseek(f, -nbytes, SEEK_END) == 0 && fread(d.data(), sizeof(double), d.size(), f) == d.size();
  fclose(f);
  if (!ok) return nfail(QGB_ERR_IO, std::string("qgb_nersc_read_host: '") + path + "' is too short");
  const uint32_t crc = crc32_update(0u, (const uint8_t*)d.data(), d.size() * sizeof(double));
  if (big == host_is_little_endian()) swap8(d);
  const uint32_t simple = simple_checksum(d);  // after the byte-order change
  for (long s = 0; s < V; ++s)
    for (int m = 0; m < 4; ++m) {
      double* u = links + (s * 4 + m) * 18;
      memcpy(u, &d[(s * 4 + m) * per_link], per_link * sizeof(double));
      if (rows == 2) memset(u + 12, 0, 6 * sizeof(double));  // rebuilt by unitarize
    }
  if (checks) *checks = (crc == h.crc ? 1 : 0) | (simple == h.simple ? 2 : 0) | (rows == 2 ? 4 : 0);
  if (file_size) *file_size = nbytes;
  return QGB_OK;
}

int qgb_save_gauge_field(const qgb_field* gf, const char* path, const char* ensemble_id, const char* ensemble_label,
                         const char* creator, double beta, int64_t sequence_num, int64_t* file_size)
{
  int32_t ts[4], mult = 0, kind = 0, prec = 0;
  int rc = qgb_field_info(gf, ts, &mult, &kind, &prec);
  if (rc != QGB_OK) return rc;
  if (kind != QGB_KIND_COLOR_MATRIX || mult != 4)
    return nfail(QGB_ERR_MISMATCH, "qgb_save_gauge_field: not a gauge field");
  const long V = volume_of(ts);
  std::vector<double> links((size_t)V * 72);
  rc = qgb_field_download(gf, links.data());
  if (rc != QGB_OK) return rc;
  double plaq = 0.0;
  rc = qgb_gf_avg_plaq(gf, &plaq);
  if (rc != QGB_OK) return rc;
  return qgb_nersc_write_host(path, links.data(), ts, plaq, link_trace_of(links.data(), V), ensemble_id,
                              ensemble_label, creator, nullptr, beta, sequence_num, file_size);
}

int qgb_load_gauge_field(qgb_field* gf, const char* path, int32_t* checks, int64_t* file_size)
{
  int32_t ts[4], mult = 0, kind = 0, prec = 0;
  int rc = qgb_field_info(gf, ts, &mult, &kind, &prec);
  if (rc != QGB_OK) return rc;
  if (kind != QGB_KIND_COLOR_MATRIX || mult != 4)
    return nfail(QGB_ERR_MISMATCH, "qgb_load_gauge_field: not a gauge field");
  const long V = volume_of(ts);
  std::vector<double> links((size_t)V * 72);
  int32_t c = 0;
  rc = qgb_nersc_read_host(path, links.data(), ts, &c, file_size);
  if (rc != QGB_OK) return rc;
  rc = qgb_field_upload(gf, links.data());
  if (rc != QGB_OK) return rc;
  if (c & 4) rc = qgb_unitarize(gf);  // two-row files: row 3 from rows 1 and 2 (qcd.h:244-246)
  if (checks) *checks = c;
  return rc;
}

}  // extern "C"
