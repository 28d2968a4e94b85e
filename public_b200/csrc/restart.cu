// Snapshot and restart files, and the direct main loop with the reference's (subset, step) restart
// semantics (src/main/cruna_hpc.f90:99-299, src/helper/io_helper.f90:11-432, src/io/hdf5_single.f90:
// 659-774).
//
// The reference writes HDF5 files: a 4-D FP64 dataset "data" (n1, n2, n3, 5), column-major, plus a
// "params" dataset of parameter strings.  libhdf5 is not available to this library, so the same
// content goes into a flat binary container with the reference's file names and a ".bin" extension:
//
//   offset  0  char[8]  magic "CRUNAB2D"
//           8  int32    version (1)
//          12  int32    element size: 8 = float64 data, 4 = int32 data
//          16  int64[4] dims (the dataset's Fortran shape; unused trailing dims are 1)
//          48  int64    length of the params text in bytes
//          56  int64    reserved (0)
//          64  params text ("key = value" lines), then the data in Fortran order
//
// restartfile.bin holds the int32 pair (ns, nt) of the last stored snapshot (cruna_hpc.f90:196-199,
// 256-259, 273-276).  Files are written to "<name>.tmp" and renamed, so an interrupted write never
// leaves a truncated restart file behind.
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cruna_internal.cuh"

namespace cruna {
void set_global_error(const std::string &msg);
}

namespace {

constexpr char kMagic[8] = {'C', 'R', 'U', 'N', 'A', 'B', '2', 'D'};

struct FileHeader {
  char magic[8];
  int32_t version;
  int32_t elem;
  int64_t dims[4];
  int64_t params_len;
  int64_t reserved;
};
static_assert(sizeof(FileHeader) == 64, "file header is 64 bytes");

int arg_fail(const std::string &msg) {
  cruna::set_global_error(msg);
  return CRUNA_ERR_ARG;
}

int io_fail(const std::string &msg) {
  cruna::set_global_error(msg);
  return CRUNA_ERR_IO;
}

int write_file(const std::string &path, int elem, const int64_t dims[4], const void *data, const std::string &params) {
  FileHeader h;
  std::memcpy(h.magic, kMagic, 8);
  h.version = 1;
  h.elem = elem;
  int64_t count = 1;
  for (int d = 0; d < 4; ++d) {
    if (dims[d] < 1) return arg_fail("snapshot dims must be >= 1");
    h.dims[d] = dims[d];
    count *= dims[d];
  }
  h.params_len = (int64_t)params.size();
  h.reserved = 0;
  const std::string tmp = path + ".tmp";
  FILE *f = std::fopen(tmp.c_str(), "wb");
  if (!f) return io_fail("cannot open " + tmp + " for writing: " + std::strerror(errno));
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  ok = ok && (params.empty() || std::fwrite(params.data(), 1, params.size(), f) == params.size());
  ok = ok && std::fwrite(data, (size_t)elem, (size_t)count, f) == (size_t)count;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    std::remove(tmp.c_str());
    return io_fail("write to " + tmp + " failed");
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) {
    std::remove(tmp.c_str());
    return io_fail("cannot rename " + tmp + " to " + path + ": " + std::strerror(errno));
  }
  return CRUNA_OK;
}

// reads the header (and the params text); leaves f positioned at the data
int open_file(const std::string &path, int elem, FileHeader &h, std::string &params, FILE *&f) {
  f = std::fopen(path.c_str(), "rb");
  if (!f) return io_fail("cannot open " + path + ": " + std::strerror(errno));
  if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1) {
    std::fclose(f);
    return io_fail(path + " is not a snapshot file of this library");
  }
  if (h.elem != elem) {
    std::fclose(f);
    return io_fail(path + " holds another element type");
  }
  if (h.params_len < 0 || h.params_len > (int64_t(1) << 24)) {
    std::fclose(f);
    return io_fail(path + ": corrupt header");
  }
  params.resize((size_t)h.params_len);
  if (h.params_len > 0 && std::fread(&params[0], 1, params.size(), f) != params.size()) {
    std::fclose(f);
    return io_fail(path + ": truncated");
  }
  return CRUNA_OK;
}

std::string fmt_int(int v, int width) {
  char b[32];
  std::snprintf(b, sizeof(b), "%0*d", width, v);
  return b;
}

// io_helper.f90:11-15 formats and the name assembly of :426-432 for the types this library writes
int make_fname(std::string &out, const char *workdir, const char *type, int world_block, int block_image, int ns,
               int nt) {
  if (!type) return arg_fail("null file type");
  const std::string wdir = std::string(workdir && *workdir ? workdir : ".") + "/";
  const std::string t(type);
  const std::string blk = "_" + fmt_int(world_block, 2), img = "_" + fmt_int(block_image, 5);
  if (t == "data_direct_snapshot" || t == "data_adjoint_snapshot")          // :146-151 / :109-114
    out = wdir + t + "_" + blk + img + "_" + fmt_int(ns, 2) + "_" + fmt_int(nt, 7);
  else if (t == "data_direct" || t == "data_adjoint")                       // :129-134 / :84-89
    out = wdir + t + "_" + blk + img + "_" + fmt_int(ns, 2);
  else if (t == "restartfile")                                              // :337-342
    out = wdir + "restartfile";
  else
    return arg_fail("unknown file type " + t);
  return CRUNA_OK;
}

std::string params_text(const cruna_config &c, int ns, int nt, int steps, int subsets) {
  char b[2048];
  std::snprintf(b, sizeof(b),
                "geom.n1 = %d\ngeom.n2 = %d\ngeom.n3 = %d\n"
                "geom.x10 = %.17g\ngeom.x20 = %.17g\ngeom.x30 = %.17g\n"
                "geom.x11 = %.17g\ngeom.x21 = %.17g\ngeom.x31 = %.17g\n"
                "material.gamma = %.17g\nmaterial.R = %.17g\nmaterial.W = %.17g\nmaterial.mu0 = %.17g\n"
                "material.T0 = %.17g\nmaterial.Pr = %.17g\n"
                "time.dt = %.17g\ntime.ns = %d\ntime.nt = %d\ntime.steps = %d\ntime.subsets = %d\n"
                "filter.alpha = %.17g\n"
                "parallelism.i1 = 1\nparallelism.i2 = 1\nparallelism.i3 = 1\n",
                c.n[0], c.n[1], c.n[2], c.x0[0], c.x0[1], c.x0[2], c.x1[0], c.x1[1], c.x1[2], c.gamma, c.R, c.W,
                c.mu0, c.T0, c.Pr, c.dt, ns, nt, steps, subsets, c.filter_alpha);
  return b;
}

}  // namespace

extern "C" {

int cruna_io_fname(char *buf, int buflen, const char *workdir, const char *type, int world_block, int block_image,
                   int ns, int nt) {
  std::string name;
  const int rc = make_fname(name, workdir, type, world_block, block_image, ns, nt);
  if (rc) return rc;
  name += ".bin";
  if (buf && buflen > 0) {
    const size_t m = std::min(name.size(), (size_t)buflen - 1);
    std::memcpy(buf, name.data(), m);
    buf[m] = 0;
  }
  return (int)name.size();
}

int cruna_write_snapshot(const char *path, const int64_t dims[4], const double *data, const char *params) {
  if (!path || !dims || !data) return arg_fail("null argument");
  return write_file(path, 8, dims, data, params ? params : "");
}

int cruna_read_snapshot(const char *path, int64_t dims[4], double *data, char *params, int params_len) {
  if (!path || !dims) return arg_fail("null argument");
  FileHeader h;
  std::string txt;
  FILE *f = nullptr;
  int rc = open_file(path, 8, h, txt, f);
  if (rc) return rc;
  int64_t count = 1;
  for (int d = 0; d < 4; ++d) {
    if (data && dims[d] != h.dims[d]) {
      std::fclose(f);
      return arg_fail(std::string(path) + ": shape differs from the expected one");
    }
    dims[d] = h.dims[d];
    count *= h.dims[d];
  }
  if (params && params_len > 0) {
    const size_t m = std::min(txt.size(), (size_t)params_len - 1);
    std::memcpy(params, txt.data(), m);
    params[m] = 0;
  }
  if (data && std::fread(data, 8, (size_t)count, f) != (size_t)count) {
    std::fclose(f);
    return io_fail(std::string(path) + ": truncated data");
  }
  std::fclose(f);
  return CRUNA_OK;
}

int cruna_write_restart(const char *workdir, int ns, int nt) {
  std::string name;
  int rc = make_fname(name, workdir, "restartfile", 1, 1, ns, nt);
  if (rc) return rc;
  const int32_t v[2] = {ns, nt};
  const int64_t dims[4] = {2, 1, 1, 1};
  return write_file(name + ".bin", 4, dims, v, "");
}

int cruna_read_restart(const char *workdir, int *ns, int *nt) {
  if (!ns || !nt) return arg_fail("null argument");
  std::string name;
  int rc = make_fname(name, workdir, "restartfile", 1, 1, 0, 0);
  if (rc) return rc;
  name += ".bin";
  FILE *probe = std::fopen(name.c_str(), "rb");
  if (!probe) return 0;                              // cruna_hpc.f90:127-131: not found, start from 0
  std::fclose(probe);
  FileHeader h;
  std::string txt;
  FILE *f = nullptr;
  rc = open_file(name, 4, h, txt, f);
  if (rc) return rc;
  int32_t v[2] = {0, 0};
  const bool ok = h.dims[0] == 2 && std::fread(v, 4, 2, f) == 2;
  std::fclose(f);
  if (!ok) return io_fail(name + ": not an (ns, nt) pair");
  *ns = v[0];
  *nt = v[1];
  return 1;
}

int cruna_restart_start(int ns, int nt, int steps, int *s0, int *nt0) {
  if (!s0 || !nt0 || steps < 1) return arg_fail("bad arguments to cruna_restart_start");
  const long long total = (long long)(ns - 1) * steps + nt + 1;      // cruna_hpc.f90:143-145
  *s0 = (int)(total / steps + 1);
  *nt0 = (int)(total - (long long)(*s0 - 1) * steps);
  return CRUNA_OK;
}

int cruna_store_snapshot(cruna_ctx *ctx, const char *workdir, const char *type, const double *q, int ns, int nt) {
  if (!ctx || !q) return arg_fail("null argument");
  const cruna_config &c = ctx->cfg;
  std::string name;
  int rc = make_fname(name, workdir, type, 1, 1, ns, nt);
  if (rc) return rc;
  const int64_t dims[4] = {c.n[0], c.n[1], c.n[2], 5};
  return write_file(name + ".bin", 8, dims, q, params_text(c, ns, nt, 0, 0));
}

int cruna_load_snapshot(cruna_ctx *ctx, const char *workdir, const char *type, double *q, int ns, int nt) {
  if (!ctx || !q) return arg_fail("null argument");
  const cruna_config &c = ctx->cfg;
  std::string name;
  int rc = make_fname(name, workdir, type, 1, 1, ns, nt);
  if (rc) return rc;
  int64_t dims[4] = {c.n[0], c.n[1], c.n[2], 5};
  return cruna_read_snapshot((name + ".bin").c_str(), dims, q, nullptr, 0);
}

int cruna_run_hpc(cruna_ctx *ctx, double *q_io, const cruna_hpc_opts *o, int *ns_out, int *nt_out) {
  if (!ctx || !q_io || !o) return arg_fail("null argument");
  if (o->steps < 1 || o->subsets < 1) return arg_fail("cruna_run_hpc: steps and subsets must be >= 1");
  const cruna_config &c = ctx->cfg;
  ctx->err.clear();
  const long long M = 5LL * c.n[0] * c.n[1] * c.n[2];
  cudaStream_t s = static_cast<cudaStream_t>(cruna_stream(ctx));
  int rc = CRUNA_OK;
  double *dq = nullptr;
  auto cuda_fail = [&](cudaError_t e) {
    ctx->err = std::string("CUDA: ") + cudaGetErrorString(e);
    cruna::set_global_error(ctx->err);
    return CRUNA_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(c.device);
  if (e == cudaSuccess) e = cudaMalloc(&dq, sizeof(double) * M);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? CRUNA_ERR_NOMEM : cuda_fail(e);
  auto store = [&](int ns, int nt, bool restartfile) -> int {
    // the device state through q_io (the caller's host array) into the snapshot file
    cudaError_t ce = cudaMemcpyAsync(q_io, dq, sizeof(double) * M, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return cuda_fail(ce);
    std::string name;
    int r = make_fname(name, o->workdir, "data_direct_snapshot", 1, 1, ns, nt);
    if (!r) {
      const int64_t dims[4] = {c.n[0], c.n[1], c.n[2], 5};
      r = write_file(name + ".bin", 8, dims, q_io, params_text(c, ns, nt, o->steps, o->subsets));
    }
    if (!r && restartfile) r = cruna_write_restart(o->workdir, ns, nt);
    return r;
  };
  const auto t_start = std::chrono::steady_clock::now();
  int ns_nt[2] = {1, 0};                                            // cruna_hpc.f90:40
  int stop_ns = 0, stop_nt = 0, stopped = 0;
  long long taken = 0;
  do {
    // initial condition (:101-103), as the reference stores it before looking for a restart
    e = cudaMemcpyAsync(dq, q_io, sizeof(double) * M, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      rc = cuda_fail(e);
      break;
    }
    if (o->dsfreq > 0 && (rc = store(1, 0, false))) break;
    if (o->restart) {                                               // :116-139
      int found = cruna_read_restart(o->workdir, &ns_nt[0], &ns_nt[1]);
      if (found < 0) {
        rc = found;
        break;
      }
      if (found == 1) {
        if ((rc = cruna_load_snapshot(ctx, o->workdir, "data_direct_snapshot", q_io, ns_nt[0], ns_nt[1]))) break;
        e = cudaMemcpyAsync(dq, q_io, sizeof(double) * M, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
          rc = cuda_fail(e);
          break;
        }
      }
    }
    int s0 = 1, nt0 = 1;
    cruna_restart_start(ns_nt[0], ns_nt[1], o->steps, &s0, &nt0);
    // the subset and step loops of :153-286; nt0 applies to every subset, as in the reference
    for (int sub = s0; sub <= o->subsets && !stopped && !rc; ++sub) {
      int nt = nt0;
      while (nt <= o->steps && !stopped && !rc) {
        // the steps up to the next event: a snapshot step, the end of the subset, the step budget,
        // or (with a wall-time limit) every step, where the reference checks its clock
        int last = o->steps;
        if (o->dsfreq > 0) last = std::min(last, ((nt + o->dsfreq - 1) / o->dsfreq) * o->dsfreq);
        if (o->walltime > 0.0) last = nt;
        if (o->max_steps > 0) last = (int)std::min<long long>(last, nt + (o->max_steps - taken) - 1);
        const int k = last - nt + 1;
        if ((rc = cruna_run_direct_dev(ctx, dq, nt - 1, k, nullptr))) break;
        taken += k;
        nt = last;
        const double elapsed =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        if ((o->walltime > 0.0 && elapsed > o->walltime) || (o->max_steps > 0 && taken >= o->max_steps)) {
          if (!(nt == o->steps && sub == o->subsets)) {             // :253-267: store and stop
            rc = store(sub, nt, true);
            stopped = 1;
            stop_ns = sub;
            stop_nt = nt;
            break;
          }
        }
        if (o->dsfreq > 0 && nt % o->dsfreq == 0 && (rc = store(sub, nt, true))) break;   // :270-278
        stop_ns = sub;
        stop_nt = nt;
        ++nt;
      }
    }
    if (rc || stopped) break;
    // last state as a snapshot (:290-291)
    if (o->dsfreq > 0) rc = store(o->subsets, o->steps, false);
  } while (false);
  if (!rc) {
    e = cudaMemcpyAsync(q_io, dq, sizeof(double) * M, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_fail(e);
  }
  cudaFree(dq);
  // file errors are reported through cruna_last_error(NULL); copy them to the context as well
  if (rc && ctx->err.empty()) ctx->err = cruna_last_error(nullptr);
  if (ns_out) *ns_out = stop_ns;
  if (nt_out) *nt_out = stop_nt;
  if (rc) return rc;
  return stopped ? CRUNA_STOPPED : CRUNA_OK;
}

}  // extern "C"
