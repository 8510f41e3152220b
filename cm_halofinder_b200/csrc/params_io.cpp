// Host side of the boundary: the run_parameters file (startup.c:109-314),
// the per-task domain of Set_Params (startup.c:33-47) and the catalog
// writers of Output_Halos / Output_Info (FOF.c:546-957).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/cmh_fof.h"

namespace cmh {
void set_error(const std::string &msg);
bool fault_active(const char *kind);  // api.cu: CMH_FAULT host-side fault injection
}

namespace {

enum TagType { kFloat, kString, kInt };

struct Tag {
  const char *name;
  TagType type;
  void *addr;
  bool seen;
};

// An output file, or NULL when it cannot be opened (or CMH_FAULT=io says so).
FILE *open_out(const char *fname) { return cmh::fault_active("io") ? nullptr : fopen(fname, "w"); }

cmh_status io_fail(const std::string &msg) {
  cmh::set_error(msg);
  return CMH_ERR_IO;
}

bool wr(const void *p, size_t size, size_t n, FILE *fp) {  // my_fwrite, main.c:95-103
  return fwrite(p, size, n, fp) == n;
}

bool wr_record(FILE *fp, const void *p, int32_t bytes) {  // Fortran record
  return wr(&bytes, 4, 1, fp) && (bytes == 0 || wr(p, 1, (size_t)bytes, fp)) &&
         wr(&bytes, 4, 1, fp);
}

}  // namespace

extern "C" {

cmh_status cmh_read_parameterfile(const char *fname, int32_t build_flags,
                                  cmh_run_parameters *out) {
  if (!fname || !out) {
    cmh::set_error("file name and output are required");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  cmh_run_parameters rp;
  memset(&rp, 0, sizeof rp);
  std::vector<Tag> tags = {
      {"Nx", kInt, &rp.Nx, false},
      {"Ny", kInt, &rp.Ny, false},
      {"Nz", kInt, &rp.Nz, false},
      {"Px", kInt, &rp.Px, false},
      {"Py", kInt, &rp.Py, false},
      {"Pz", kInt, &rp.Pz, false},
      {"Lxmin", kFloat, &rp.Lxmin, false},
      {"Lymin", kFloat, &rp.Lymin, false},
      {"Lzmin", kFloat, &rp.Lzmin, false},
      {"Lxmax", kFloat, &rp.Lxmax, false},
      {"Lymax", kFloat, &rp.Lymax, false},
      {"Lzmax", kFloat, &rp.Lzmax, false},
      {"Seed", kInt, &rp.Seed, false},
      {"Buffer", kFloat, &rp.Buffer, false},
      {"Boundarysize", kFloat, &rp.Boundarysize, false},
      {"Linklength", kFloat, &rp.Linklength, false},
      {"Nphalomin", kFloat, &rp.Nphalomin, false},
      {"SampInHalos", kFloat, &rp.SampInHalos, false},
      {"SampOutHalos", kFloat, &rp.SampOutHalos, false},
      {"InputStyle", kInt, &rp.InputStyle, false},
      {"Ninputfiles", kInt, &rp.Ninputfiles, false},
      {"Starting_file", kInt, &rp.Starting_file, false},
      {"Nread", kInt, &rp.Nread, false},
      {"Nwrite", kInt, &rp.Nwrite, false},
      {"InputFileBase", kString, rp.InputFileBase, false},
      {"OutputFileBase", kString, rp.OutputFileBase, false},
  };
  if (build_flags & CMH_TAGS_INFOFILE) tags.push_back({"InputInfoFile", kString, rp.InputInfoFile, false});
  if (build_flags & CMH_TAGS_VARLINK) {
    tags.push_back({"Omega", kFloat, &rp.Omega, false});
    tags.push_back({"Origin_x", kFloat, &rp.Origin_x, false});
    tags.push_back({"Origin_y", kFloat, &rp.Origin_y, false});
    tags.push_back({"Origin_z", kFloat, &rp.Origin_z, false});
  }
  std::string errors;
  FILE *fd = fopen(fname, "r");
  if (!fd) {
    cmh::set_error(std::string("Parameter file ") + fname + " not found.");
    return CMH_ERR_PARAMETER_FILE;
  }
  char buf[500], b1[500], b2[500], b3[500];
  while (fgets(buf, sizeof buf, fd)) {
    if (sscanf(buf, "%499s%499s%499s", b1, b2, b3) < 2) continue;
    if (b1[0] == '%') continue;
    Tag *t = nullptr;
    for (Tag &c : tags)
      if (!c.seen && strcmp(b1, c.name) == 0) {
        t = &c;
        break;
      }
    if (!t) {
      errors += std::string("Tag '") + b1 + "' not allowed or multiple defined. ";
      continue;
    }
    t->seen = true;
    switch (t->type) {
      case kFloat: *static_cast<double *>(t->addr) = atof(b2); break;
      case kInt: *static_cast<int32_t *>(t->addr) = atoi(b2); break;
      case kString:
        strncpy(static_cast<char *>(t->addr), b2, 499);
        static_cast<char *>(t->addr)[499] = 0;
        break;
    }
  }
  fclose(fd);
  for (const Tag &c : tags)
    if (!c.seen) errors += std::string("I miss a value for tag '") + c.name + "'. ";
  if (!errors.empty()) {
    cmh::set_error(std::string("in run parameters file ") + fname + ": " + errors);
    return CMH_ERR_PARAMETER_FILE;
  }
  *out = rp;
  return CMH_OK;
}

cmh_status cmh_params_from_run(const cmh_run_parameters *rp, int32_t task, int32_t periodic,
                               cmh_fof_params *out) {
  if (!rp || !out) {
    cmh::set_error("run parameters and output are required");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  const int ntask = rp->Nx * rp->Ny * rp->Nz;
  if (rp->Nx <= 0 || rp->Ny <= 0 || rp->Nz <= 0 || task < 0 || task >= ntask) {
    cmh::set_error("task outside the Nx*Ny*Nz task grid (startup.c:13-16)");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  const int lz = task / (rp->Nx * rp->Ny);
  const int ly = (task - rp->Nx * rp->Ny * lz) / rp->Nx;
  const int lx = task - rp->Nx * ly - rp->Nx * rp->Ny * lz;
  const double Lmin[3] = {rp->Lxmin, rp->Lymin, rp->Lzmin};
  const double Lmax[3] = {rp->Lxmax, rp->Lymax, rp->Lzmax};
  const int N[3] = {rp->Nx, rp->Ny, rp->Nz}, l[3] = {lx, ly, lz};
  cmh_fof_params p;
  memset(&p, 0, sizeof p);
  for (int a = 0; a < 3; a++) {
    p.lo[a] = l[a] * ((Lmax[a] - Lmin[a]) / (double)N[a]) + Lmin[a];
    p.hi[a] = p.lo[a] + ((Lmax[a] - Lmin[a]) / (double)N[a]);
    p.ref_cells[a] = (a == 0 ? rp->Px : a == 1 ? rp->Py : rp->Pz);
  }
  p.boundary = rp->Boundarysize;
  p.linklength = rp->Linklength;
  p.nphalomin = rp->Nphalomin;
  p.periodic = periodic ? 1 : 0;
  p.precision = CMH_FP32_RECHECK;
  p.origin[0] = rp->Origin_x;
  p.origin[1] = rp->Origin_y;
  p.origin[2] = rp->Origin_z;
  *out = p;
  return CMH_OK;
}

cmh_status cmh_write_halos(const char *base, int32_t task, const cmh_catalog *cat,
                           const cmh_particles *parts, uint32_t flags) {
  if (!base || !cat || (cat->nhalos > 0 && (!cat->props || cat->location != CMH_HOST))) {
    cmh::set_error("a host catalog is required");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  const bool unf = flags & CMH_OUT_UNFORMATTED, withp = flags & CMH_OUT_PARTICLES,
             withid = flags & CMH_OUT_PARTICLE_ID;
  const int64_t nh = cat->nhalos;
  const int hs = cat->halosize;
  if (nh <= 0) return CMH_OK;  // FOF.c:588: no file without halos
  if (nh > 0x7fffffffll) {
    cmh::set_error("more halos than the catalog's int header can hold");
    return CMH_ERR_CAPACITY;
  }
  const int64_t n_in = cat->stats.n_in;
  std::vector<int64_t> order;    // members grouped by halo
  std::vector<int64_t> mstart;
  if (withp) {
    if (!cat->member || !cat->member_proc || !cat->member_pos || !parts || !parts->vel ||
        parts->location != CMH_HOST || parts->n != n_in || (withid && !parts->id)) {
      cmh::set_error("particle output needs host members, velocities (and IDs)");
      return CMH_ERR_INVALID_ARGUMENT;
    }
    mstart.assign(nh + 1, 0);
    for (int64_t i = 0; i < n_in; i++)
      if (cat->member[i] >= 0 && cat->member[i] < nh) mstart[cat->member[i] + 1]++;
    std::partial_sum(mstart.begin(), mstart.end(), mstart.begin());
    order.resize(mstart[nh]);
    std::vector<int64_t> fill(mstart.begin(), mstart.end() - 1);
    for (int64_t i = 0; i < n_in; i++)
      if (cat->member[i] >= 0 && cat->member[i] < nh) order[fill[cat->member[i]]++] = i;
    for (int64_t h = 0; h < nh; h++)
      std::sort(order.begin() + mstart[h], order.begin() + mstart[h + 1],
                [&](int64_t a, int64_t b) { return cat->member_proc[a] < cat->member_proc[b]; });
  }
  char fname[1100];
  snprintf(fname, sizeof fname, "%s.%d", base, task);
  FILE *fp = open_out(fname);
  if (!fp) return io_fail(std::string("Unable to open output file ") + fname);
  bool ok = true;
  const int32_t nhi = (int32_t)nh;
  auto vel_of = [&](int64_t i, int a) -> float {
    return parts->vel_dtype == CMH_FLOAT64 ? (float)((const double *)parts->vel)[3 * i + a]
                                           : ((const float *)parts->vel)[3 * i + a];
  };
  if (withp) {
    if (unf) ok &= wr_record(fp, &nhi, 4);
    else ok &= fprintf(fp, "%15d\n", nhi) > 0;
    for (int64_t h = 0; h < nh && ok; h++) {
      const float *rec = cat->props + h * hs;
      if (unf) {
        ok &= wr_record(fp, rec, (int32_t)(sizeof(float) * hs));
      } else {
        fprintf(fp, "%15d", (int)rec[0]);
        for (int q = 1; q < hs; q++) fprintf(fp, " %15.6f", rec[q]);
        ok &= fprintf(fp, "\n") > 0;
      }
      for (int64_t m = mstart[h]; m < mstart[h + 1] && ok; m++) {
        const int64_t i = order[m];
        float pv[6] = {cat->member_pos[3 * i], cat->member_pos[3 * i + 1],
                       cat->member_pos[3 * i + 2], vel_of(i, 0), vel_of(i, 1), vel_of(i, 2)};
        if (unf) {
          int32_t d = (int32_t)(sizeof pv + (withid ? 8 : 0));
          ok &= wr(&d, 4, 1, fp);
          if (withid) ok &= wr(&parts->id[i], 8, 1, fp);
          ok &= wr(pv, sizeof pv, 1, fp) && wr(&d, 4, 1, fp);
        } else if (withid) {
          ok &= fprintf(fp, "%15llu %15.6f %15.6f %15.6f %15.6f %15.6f %15.6f\n",
                        (unsigned long long)parts->id[i], pv[0], pv[1], pv[2], pv[3], pv[4],
                        pv[5]) > 0;
        } else {
          ok &= fprintf(fp, "%15.6f %15.6f %15.6f %15.6f %15.6f %15.6f\n", pv[0], pv[1], pv[2],
                        pv[3], pv[4], pv[5]) > 0;
        }
      }
    }
  } else if (unf) {
    // one record with every halo (FOF.c:781-790,873-881)
    ok &= wr_record(fp, &nhi, 4);
    const int64_t bytes = nh * hs * (int64_t)sizeof(float);
    if (bytes > 0x7fffffffll) {
      fclose(fp);
      cmh::set_error("halo block larger than a Fortran record");
      return CMH_ERR_CAPACITY;
    }
    ok &= wr_record(fp, cat->props, (int32_t)bytes);
  } else {
    // one line per halo; the dispersion-only layout prints the dispersion
    // values (the reference's FOF.c:895-896 indexes them past the block)
    for (int64_t h = 0; h < nh && ok; h++) {
      const float *rec = cat->props + h * hs;
      fprintf(fp, "%15d", (int)rec[0]);
      for (int q = 1; q < hs; q++) fprintf(fp, " %15.6f", rec[q]);
      ok &= fprintf(fp, "\n") > 0;
    }
  }
  ok &= fclose(fp) == 0;
  if (!ok) return io_fail(std::string("I/O error writing ") + fname);
  return CMH_OK;
}

cmh_status cmh_write_info_sampled(const char *base, const cmh_run_parameters *rp,
                                  const int64_t *nhalos_per_task,
                                  const int64_t *ninhalo_per_task,
                                  const int64_t *nouthalo_per_task, int32_t ntask) {
  if (!base || !rp || (ntask > 0 && !nhalos_per_task) || ntask != rp->Nx * rp->Ny * rp->Nz) {
    cmh::set_error("info file needs one halo count per task of the Nx*Ny*Nz grid");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  char fname[1100];
  snprintf(fname, sizeof fname, "%s.info", base);
  FILE *fp = open_out(fname);
  if (!fp) return io_fail(std::string("Can't write in file ") + fname);
  fprintf(fp, "#    FILENUM      XMIN         YMIN        ZMIN         XMAX         YMAX         ZMAX         NHALOS     NSUBSAMPIN     NSUBSAMPOUT    \n");
  const int Nx = rp->Nx, Ny = rp->Ny, Nz = rp->Nz;
  for (int i = 0; i < ntask; i++) {
    const int tz = i / (Nx * Ny), ty = (i - Nx * Ny * tz) / Nx, tx = i - Nx * ty - Nx * Ny * tz;
    const double x0 = tx * ((rp->Lxmax - rp->Lxmin) / (double)Nx) + rp->Lxmin;
    const double y0 = ty * ((rp->Lymax - rp->Lymin) / (double)Ny) + rp->Lymin;
    const double z0 = tz * ((rp->Lzmax - rp->Lzmin) / (double)Nz) + rp->Lzmin;
    const double x1 = x0 + ((rp->Lxmax - rp->Lxmin) / (double)Nx);
    const double y1 = y0 + ((rp->Lymax - rp->Lymin) / (double)Ny);
    const double z1 = z0 + ((rp->Lzmax - rp->Lzmin) / (double)Nz);
    const unsigned nin = ninhalo_per_task ? (unsigned)ninhalo_per_task[i] : 0u;
    const unsigned nout = nouthalo_per_task ? (unsigned)nouthalo_per_task[i] : 0u;
    fprintf(fp, "%12d %12.6lf %12.6lf %12.6lf %12.6lf %12.6lf %12.6lf %12d %12u %12u\n", i, x0,
            y0, z0, x1, y1, z1, (int)nhalos_per_task[i], nin, nout);
  }
  if (fclose(fp) != 0) return io_fail(std::string("I/O error writing ") + fname);
  return CMH_OK;
}

cmh_status cmh_write_info(const char *base, const cmh_run_parameters *rp,
                          const int64_t *nhalos_per_task, int32_t ntask) {
  return cmh_write_info_sampled(base, rp, nhalos_per_task, nullptr, nullptr, ntask);
}

cmh_status cmh_write_subsample(const char *base, int32_t task, int32_t in,
                               const cmh_particles *parts, const int64_t *idx, int64_t n,
                               uint32_t flags) {
  const bool unf = flags & CMH_OUT_UNFORMATTED, withid = flags & CMH_OUT_PARTICLE_ID;
  if (!base || n < 0 || (n > 0 && (!idx || !parts || !parts->pos || !parts->vel ||
                                    parts->location != CMH_HOST || (withid && !parts->id)))) {
    cmh::set_error("a subsample needs host positions, velocities (and IDs) and its indices");
    return CMH_ERR_INVALID_ARGUMENT;
  }
  if (n == 0) return CMH_OK;  // FOF.c:457: no file for an empty sample
  for (int64_t k = 0; k < n; k++)
    if (idx[k] < 0 || idx[k] >= parts->n) {
      cmh::set_error("subsample index outside the particles");
      return CMH_ERR_INVALID_ARGUMENT;
    }
  if (n > 0x7fffffffll / 12) {
    cmh::set_error("subsample larger than a Fortran record");
    return CMH_ERR_CAPACITY;
  }
  auto val = [&](const void *a, int dtype, int64_t i, int c) -> float {
    return dtype == CMH_FLOAT64 ? (float)((const double *)a)[3 * i + c]
                                : ((const float *)a)[3 * i + c];
  };
  char fname[1100];
  snprintf(fname, sizeof fname, "%s_%s.%d", base, in ? "inhalo" : "outhalo", task);
  FILE *fp = open_out(fname);
  if (!fp) return io_fail(std::string("Unable to open output file ") + fname);
  bool ok = true;
  if (unf) {
    const uint32_t nn = (uint32_t)n;
    ok &= wr_record(fp, &nn, 4);
    std::vector<float> block((size_t)n * 3);
    for (int q = 0; q < 2 && ok; q++) {
      const void *a = q == 0 ? parts->pos : parts->vel;
      const int dt = q == 0 ? parts->pos_dtype : parts->vel_dtype;
      for (int64_t k = 0; k < n; k++)
        for (int c = 0; c < 3; c++) block[3 * k + c] = val(a, dt, idx[k], c);
      ok &= wr_record(fp, block.data(), (int32_t)(sizeof(float) * 3 * n));
    }
    if (withid && ok) {
      std::vector<uint64_t> ids((size_t)n);
      for (int64_t k = 0; k < n; k++) ids[k] = parts->id[idx[k]];
      if (n > 0x7fffffffll / 8) ok = false;
      else ok &= wr_record(fp, ids.data(), (int32_t)(sizeof(uint64_t) * n));
    }
  } else {
    for (int64_t k = 0; k < n && ok; k++) {
      const int64_t i = idx[k];
      const float pv[6] = {val(parts->pos, parts->pos_dtype, i, 0),
                           val(parts->pos, parts->pos_dtype, i, 1),
                           val(parts->pos, parts->pos_dtype, i, 2),
                           val(parts->vel, parts->vel_dtype, i, 0),
                           val(parts->vel, parts->vel_dtype, i, 1),
                           val(parts->vel, parts->vel_dtype, i, 2)};
      if (withid)
        ok &= fprintf(fp, "%15llu %15.6f %15.6f %15.6f %15.6f %15.6f %15.6f\n",
                      (unsigned long long)parts->id[i], pv[0], pv[1], pv[2], pv[3], pv[4],
                      pv[5]) > 0;
      else
        ok &= fprintf(fp, "%15.6f %15.6f %15.6f %15.6f %15.6f %15.6f\n", pv[0], pv[1], pv[2],
                      pv[3], pv[4], pv[5]) > 0;
    }
  }
  ok &= fclose(fp) == 0;
  if (!ok) return io_fail(std::string("I/O error writing ") + fname);
  return CMH_OK;
}

}  // extern "C"
