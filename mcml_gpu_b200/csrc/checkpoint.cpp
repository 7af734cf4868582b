// checkpoint.cpp -- the checkpoint file of a chunked first pass (host only).
//
// Layout (little-endian), declared with mcml_run_checkpointed in
// include/mcml_b200.h: a 128-byte header, then the detection records in
// the order they were appended.  Updates are append-then-header: the new
// records go after the ones the header counts and are flushed to disk
// before the header that counts them is rewritten, so an interrupted
// update leaves the previous checkpoint intact (trailing bytes beyond the
// counted records are ignored and overwritten by the next update).
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "internal.h"

namespace mcml {

namespace {

constexpr char kMagic[8] = {'M', 'C', 'M', 'L', 'C', 'K', 'P', '1'};
constexpr uint32_t kVersion = 1;
constexpr size_t kDigestSpan = 96;  // header bytes covered by header_digest
static_assert(sizeof(CkptHeader) == 128, "checkpoint header layout");
static_assert(offsetof(CkptHeader, header_digest) == kDigestSpan, "checkpoint header layout");

bool write_all(int fd, const void *p, size_t n, off_t off) {
  const char *c = static_cast<const char *>(p);
  while (n) {
    const ssize_t w = pwrite(fd, c, n, off);
    if (w <= 0) return false;
    c += w;
    n -= (size_t)w;
    off += w;
  }
  return true;
}

bool read_all(int fd, void *p, size_t n, off_t off) {
  char *c = static_cast<char *>(p);
  while (n) {
    const ssize_t r = pread(fd, c, n, off);
    if (r <= 0) return false;
    c += r;
    n -= (size_t)r;
    off += r;
  }
  return true;
}

}  // namespace

uint64_t fnv1a(const void *p, size_t n, uint64_t h) {
  const unsigned char *c = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}

// Digest of what determines a run's photons: the simulation's used fields
// and the slot layout (not the chunking, which changes nothing).
uint64_t run_digest(const mcml_sim &s, uint64_t seed, uint64_t slot_begin, uint64_t slots) {
  uint64_t h = kFnvBasis;
  auto add = [&](const void *p, size_t n) { h = fnv1a(p, n, h); };
  add(&s.number_photons, 8);
  add(&s.num_layers, 4);
  add(&s.num_sds, 4);
  add(&s.upper_n, 4);
  add(&s.lower_n, 4);
  add(&s.detector_reflectance, 4);
  add(&s.source_probe_oblique, 4);
  add(&s.detector_probe_oblique, 4);
  add(&s.source_NA, 4);
  add(&s.source_radius, 4);
  add(&s.source_angle_deg, 4);
  const uint32_t S = s.num_sds < MCML_MAX_SDS ? s.num_sds : MCML_MAX_SDS;
  const uint32_t L = s.num_layers < MCML_MAX_LAYERS ? s.num_layers : MCML_MAX_LAYERS;
  add(s.det_pos, 4 * S);
  add(s.det_NA, 4 * S);
  add(s.det_radius, 4 * S);
  add(s.det_angle_deg, 4 * S);
  add(s.height, 4 * L);
  add(s.mua, 4 * L);
  add(s.mus, 4 * L);
  add(s.n, 4 * L);
  add(s.g, 4 * L);
  add(&seed, 8);
  add(&slot_begin, 8);
  add(&slots, 8);
  return h;
}

void ckpt_init(CkptHeader &h) {
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.record_bytes = kRecordBytes;
  h.records_digest = kFnvBasis;
}

int ckpt_read_header(const std::string &path, CkptHeader &h, bool &exists) {
  exists = false;
  const int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) return MCML_OK;  // no checkpoint yet
  exists = true;
  const bool ok = read_all(fd, &h, sizeof(h), 0);
  const off_t size = lseek(fd, 0, SEEK_END);
  close(fd);
  if (!ok) return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": short header");
  if (std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion ||
      h.record_bytes != kRecordBytes)
    return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": not a version-1 checkpoint");
  if (fnv1a(&h, kDigestSpan, kFnvBasis) != h.header_digest)
    return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": header digest mismatch");
  if (h.slots_done > h.slots)
    return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": slots_done beyond slots");
  if ((uint64_t)size < sizeof(h) + h.records * (uint64_t)kRecordBytes)
    return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": truncated records");
  return MCML_OK;
}

int ckpt_read_records(const std::string &path, const CkptHeader &h, void *dst) {
  const int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) return set_error(MCML_E_IO, "cannot open " + path);
  const size_t n = (size_t)h.records * kRecordBytes;
  const bool ok = n == 0 || read_all(fd, dst, n, (off_t)sizeof(h));
  close(fd);
  if (!ok) return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": truncated records");
  if (fnv1a(dst, n, kFnvBasis) != h.records_digest)
    return set_error(MCML_E_CHECKPOINT, "checkpoint " + path + ": record digest mismatch");
  return MCML_OK;
}

int ckpt_write_header(const std::string &path, CkptHeader &h) {
  const int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) return set_error(MCML_E_IO, "cannot open " + path + " for writing");
  h.header_digest = fnv1a(&h, kDigestSpan, kFnvBasis);
  const bool ok = write_all(fd, &h, sizeof(h), 0) && fsync(fd) == 0;
  close(fd);
  return ok ? MCML_OK : set_error(MCML_E_IO, "cannot write checkpoint " + path);
}

int ckpt_append(const std::string &path, CkptHeader &h, const void *recs, uint64_t n,
                uint64_t slots_done, uint64_t steps) {
  const int fd = open(path.c_str(), O_WRONLY | O_CREAT, 0644);
  if (fd < 0) return set_error(MCML_E_IO, "cannot open " + path + " for writing");
  const size_t bytes = (size_t)n * kRecordBytes;
  const off_t off = (off_t)(sizeof(h) + h.records * (uint64_t)kRecordBytes);
  bool ok = bytes == 0 || write_all(fd, recs, bytes, off);
  ok = ok && fsync(fd) == 0;
  if (ok) {
    CkptHeader next = h;
    next.records = h.records + n;
    next.records_digest = fnv1a(recs, bytes, h.records_digest);
    next.slots_done = slots_done;
    next.steps = steps;
    next.launches = h.launches + 1;
    next.header_digest = fnv1a(&next, kDigestSpan, kFnvBasis);
    ok = write_all(fd, &next, sizeof(next), 0) && fsync(fd) == 0;
    if (ok) h = next;
  }
  close(fd);
  return ok ? MCML_OK : set_error(MCML_E_IO, "cannot write checkpoint " + path);
}

}  // namespace mcml

using namespace mcml;

extern "C" int mcml_checkpoint_read_info(const char *path, mcml_checkpoint_info *info) {
  clear_error();
  if (!path || !info) return set_error(MCML_E_INVALID, "null argument");
  CkptHeader h;
  bool exists = false;
  int rc = ckpt_read_header(path, h, exists);
  if (rc) return rc;
  if (!exists) return set_error(MCML_E_IO, std::string("cannot open ") + path);
  info->seed = h.seed;
  info->slot_begin = h.slot_begin;
  info->photons = h.photons;
  info->slots = h.slots;
  info->slots_done = h.slots_done;
  info->records = h.records;
  info->steps = h.steps;
  info->launches = h.launches;
  return MCML_OK;
}
