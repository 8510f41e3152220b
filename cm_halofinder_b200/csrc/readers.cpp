// Particle readers: the input formats of Read_Data (read_data.c:100-404) --
// ASCII lines, Gadget-1 snapshot files (GADGET_STYLE) and PICOLA unformatted
// lightcone files (LIGHTCONE + UNFORMATTED) -- for one process that reads
// every file of a run.  Each reader appends the file's particles in file
// order; the domain filter and the ghost images are the FoF run's business.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cmh_fof.h"

namespace cmh {
bool fault_active(const char *kind);  // api.cu: CMH_FAULT host-side fault injection
void set_error(const std::string &msg);
}

namespace {

struct Fail {
  cmh_status code;
  std::string msg;
};

[[noreturn]] void fail(cmh_status code, const std::string &msg) { throw Fail{code, msg}; }

// Accumulates the particles of all files; positions and velocities in
// float or double, IDs widened to 64 bits.
struct Sink {
  bool f64 = false, with_id = false;
  std::vector<float> pf, vf;
  std::vector<double> pd, vd;
  std::vector<uint64_t> id;
  int64_t n = 0;
  void add(const double *x, const double *v, uint64_t ident) {
    for (int a = 0; a < 3; a++) {
      if (f64) {
        pd.push_back(x[a]);
        vd.push_back(v[a]);
      } else {
        pf.push_back((float)x[a]);
        vf.push_back((float)v[a]);
      }
    }
    if (with_id) id.push_back(ident);
    n++;
  }
  void addf(const float *x, const float *v, uint64_t ident) {
    for (int a = 0; a < 3; a++) {
      pf.push_back(x[a]);
      vf.push_back(v[a]);
    }
    if (with_id) id.push_back(ident);
    n++;
  }
};

struct File {
  FILE *fp = nullptr;
  std::string name;
  File(const std::string &n, const char *mode) : name(n) {
    fp = cmh::fault_active("io") ? nullptr : fopen(n.c_str(), mode);
    if (!fp) fail(CMH_ERR_IO, "unable to open file " + n);
  }
  ~File() {
    if (fp) fclose(fp);
  }
  // my_fread (main.c:83-91): a short read is an I/O error
  void read(void *p, size_t size, size_t n) {
    if (fread(p, size, n, fp) != n) fail(CMH_ERR_IO, "I/O error (fread) on file " + name);
  }
};

// ASCII (read_data.c:276-315 and 368-404): the file's line count is its
// particle count; each particle is "[ID] x y z vx vy vz", the values read
// with the precision of the build (float in MEMORY_MODE).
void read_ascii(const std::string &name, Sink &out) {
  File f(name, "r");
  int64_t lines = 0;
  char buf[500];
  while (fgets(buf, sizeof buf, f.fp)) lines++;  // as the reference counts them
  rewind(f.fp);
  std::string text;
  {
    std::vector<char> all;
    char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof chunk, f.fp)) > 0) all.insert(all.end(), chunk, chunk + got);
    text.assign(all.begin(), all.end());
  }
  const char *p = text.c_str();
  auto bad = [&]() { fail(CMH_ERR_IO, "incorrect line format in file " + name); };
  for (int64_t j = 0; j < lines; j++) {
    uint64_t ident = 0;
    char *end = nullptr;
    if (out.with_id) {
      errno = 0;
      ident = strtoull(p, &end, 10);
      if (end == p || errno) bad();
      p = end;
    }
    double x[3], v[3];
    float xf[3], vf[3];
    for (int c = 0; c < 6; c++) {
      if (out.f64) {
        const double d = strtod(p, &end);
        if (end == p) bad();
        (c < 3 ? x[c] : v[c - 3]) = d;
      } else {
        const float fl = strtof(p, &end);
        if (end == p) bad();
        (c < 3 ? xf[c] : vf[c - 3]) = fl;
      }
      p = end;
    }
    if (out.f64) out.add(x, v, ident);
    else out.addf(xf, vf, ident);
  }
}

// Gadget-1 snapshot (read_data.c:321-365): a 256-byte header record whose
// npart[1] counts the particles, then position, velocity and (PARTICLE_ID)
// 64-bit ID records, each framed by 4-byte record lengths.
void read_gadget(const std::string &name, Sink &out) {
  File f(name, "rb");
  int32_t dummy;
  unsigned char header[256];
  f.read(&dummy, 4, 1);
  f.read(header, sizeof header, 1);
  f.read(&dummy, 4, 1);
  uint32_t npart[6];
  memcpy(npart, header, sizeof npart);
  const size_t n = npart[1];
  std::vector<float> pos(3 * n), vel(3 * n);
  std::vector<uint64_t> ids(n, 0);
  f.read(&dummy, 4, 1);
  if (n) f.read(pos.data(), sizeof(float), 3 * n);
  f.read(&dummy, 4, 1);
  f.read(&dummy, 4, 1);
  if (n) f.read(vel.data(), sizeof(float), 3 * n);
  f.read(&dummy, 4, 1);
  if (out.with_id) {
    f.read(&dummy, 4, 1);
    if (n) f.read(ids.data(), sizeof(uint64_t), n);
    f.read(&dummy, 4, 1);
  }
  for (size_t j = 0; j < n; j++) {
    if (out.f64) {
      const double x[3] = {pos[3 * j], pos[3 * j + 1], pos[3 * j + 2]};
      const double v[3] = {vel[3 * j], vel[3 * j + 1], vel[3 * j + 2]};
      out.add(x, v, ids[j]);
    } else {
      out.addf(&pos[3 * j], &vel[3 * j], ids[j]);
    }
  }
}

// PICOLA unformatted lightcone (read_data.c:212-273): blocks of
// [4][npart][4] [4] npart x ([32-bit ID] x y z vx vy vz as float) [4]
// until the end of the file.  The reference reads the 32-bit ID into a
// 64-bit variable; here it is zero-extended.
void read_picola(const std::string &name, Sink &out) {
  File f(name, "rb");
  while (true) {
    int32_t dummy;
    if (fread(&dummy, 4, 1, f.fp) != 1) break;  // end of the file
    uint32_t npart = 0;
    f.read(&npart, sizeof npart, 1);
    f.read(&dummy, 4, 1);
    f.read(&dummy, 4, 1);
    for (uint32_t j = 0; j < npart; j++) {
      uint32_t ident = 0;
      if (out.with_id) f.read(&ident, sizeof ident, 1);
      float x[3], v[3];
      f.read(x, sizeof(float), 3);
      f.read(v, sizeof(float), 3);
      if (out.f64) {
        const double xd[3] = {x[0], x[1], x[2]}, vd[3] = {v[0], v[1], v[2]};
        out.add(xd, vd, ident);
      } else {
        out.addf(x, v, ident);
      }
    }
    f.read(&dummy, 4, 1);
  }
}

// The run's input files (read_data.c:100-124, 178-198): InputStyle 0 reads
// "<InputFileBase>.<n>" for n = Starting_file .. Starting_file+Ninputfiles-1;
// otherwise InputFileBase lists one file per line (blank lines and lines
// starting with '%' skipped).
std::vector<std::string> input_files(const cmh_run_parameters &rp) {
  std::vector<std::string> files;
  if (rp.InputStyle == 0) {
    for (int i = 0; i < rp.Ninputfiles; i++)
      files.push_back(std::string(rp.InputFileBase) + "." + std::to_string(i + rp.Starting_file));
    return files;
  }
  File list(rp.InputFileBase, "rb");
  char buf[500];
  while (fgets(buf, sizeof buf, list.fp)) {
    char b1[500], b2[500];
    if (sscanf(buf, "%499s%499s", b1, b2) < 1) continue;
    if (b1[0] == '%') continue;
    files.emplace_back(b1);
  }
  return files;
}

}  // namespace

struct cmh_particle_store {
  std::vector<float> pf, vf;
  std::vector<double> pd, vd;
  std::vector<uint64_t> id;
};

extern "C" {

cmh_status cmh_read_particles(const cmh_run_parameters *rp, int32_t format, uint32_t flags,
                              cmh_particles *out, cmh_particle_store **store) {
  if (!rp || !out || !store) {
    cmh::set_error("run parameters, particles and store are required");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  memset(out, 0, sizeof *out);
  *store = nullptr;
  try {
    if (format != CMH_FMT_ASCII && format != CMH_FMT_GADGET1 &&
        format != CMH_FMT_PICOLA_LIGHTCONE)
      fail(CMH_ERR_INVALID_ARGUMENT, "unknown input format");
    Sink sink;
    sink.with_id = (flags & CMH_READ_PARTICLE_ID) != 0;
    sink.f64 = (flags & CMH_READ_FP64) != 0;
    for (const std::string &name : input_files(*rp)) {
      if (format == CMH_FMT_ASCII) read_ascii(name, sink);
      else if (format == CMH_FMT_GADGET1) read_gadget(name, sink);
      else read_picola(name, sink);
    }
    cmh_particle_store *own = new cmh_particle_store;
    own->pf.swap(sink.pf);
    own->vf.swap(sink.vf);
    own->pd.swap(sink.pd);
    own->vd.swap(sink.vd);
    own->id.swap(sink.id);
    out->n = sink.n;
    out->pos_dtype = out->vel_dtype = sink.f64 ? CMH_FLOAT64 : CMH_FLOAT32;
    out->pos = sink.f64 ? (const void *)own->pd.data() : (const void *)own->pf.data();
    out->vel = sink.f64 ? (const void *)own->vd.data() : (const void *)own->vf.data();
    out->id = sink.with_id ? own->id.data() : nullptr;
    out->location = CMH_HOST;
    *store = own;
  } catch (const Fail &e) {
    cmh::set_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    cmh::set_error("host memory exhausted while reading particles");
    return CMH_ERR_OUT_OF_MEMORY;
  }
  return CMH_OK;
}

void cmh_particle_store_free(cmh_particle_store *store) { delete store; }

}  // extern "C"
