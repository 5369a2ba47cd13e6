// output.cu -- the on-disk formats around the step: the VTK image-data files of
// source/output/pmlib_output_mesh.f, the topology summary of
// source/output/pmlib_output_topology.f, and the vortex client's particle restart
// file (vortex_codes/vortex_structures/source/output/output_particles.f, read back
// as input/input_particles.f reads it).  Host code; device arrays are copied to the
// host first.  The bytes follow what the reference's gfortran build writes: the
// .pvti is formatted text, the .vti an unformatted stream (strings without line
// ends, raw little-endian numbers), the restart file unformatted sequential
// (every record framed by its 4-byte length).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pmlib_gpu.h"

namespace pmgpu {
void set_error(const char *caller, const char *msg);  // pmgpu.cu: message format of source/pmlib_write.f
}
using pmgpu::set_error;

namespace {

// Fortran Iw
std::string fmt_i(long long v, int w) {
  char b[64];
  snprintf(b, sizeof(b), "%*lld", w, v);
  return b;
}

// Fortran Ew.d (0.dddE+ee, d significant digits, right-justified in w)
std::string fmt_e(double x, int w, int d) {
  char m[80];
  if (x == 0.0) {
    std::string s = "0." + std::string(d, '0') + "E+00";
    return std::string(w > (int)s.size() ? w - (int)s.size() : 0, ' ') + s;
  }
  snprintf(m, sizeof(m), "%.*e", d - 1, std::fabs(x));  // d.ddd...e+ee, correctly rounded
  std::string ms(m);
  const size_t ep = ms.find('e');
  std::string digits = ms.substr(0, 1) + ms.substr(2, ep - 2);
  const int e10 = atoi(ms.c_str() + ep + 1) + 1;
  char ex[16];
  if (std::abs(e10) < 100) snprintf(ex, sizeof(ex), "E%c%02d", e10 < 0 ? '-' : '+', std::abs(e10));
  else snprintf(ex, sizeof(ex), "%c%03d", e10 < 0 ? '-' : '+', std::abs(e10));
  std::string s = std::string(x < 0 ? "-" : "") + "0." + digits + ex;
  return std::string(w > (int)s.size() ? w - (int)s.size() : 0, ' ') + s;
}

std::string extent6(const int *icell, const int *ncell) {
  std::string s;
  for (int d = 0; d < 3; d++) s += fmt_i(icell[d] - 1, 8) + fmt_i(icell[d] + ncell[d] - 1, 8);
  return s;
}

std::string origin_spacing(const pmgpu_patch *p) {
  std::string s = "\" Ghostlevel=\"0\" Origin=\"";
  for (int d = 0; d < 3; d++) s += fmt_e(p->xmin[d], 20, 12);
  s += "\" Spacing=\"";
  for (int d = 0; d < 3; d++) s += fmt_e(p->dx[d], 20, 12);
  return s + "\">";
}

// interior values (c, i, j, k) of a mesh as float32, in the reference's loop order
int interior_f32(const pmgpu_topo *t, int precision, const void *mesh, int device, std::vector<float> &out,
                 const char *caller) {
  int ext[3];
  size_t npt = 1;
  for (int d = 0; d < 3; d++) {
    ext[d] = t->ncell[d] + t->nghost[2 * d] + t->nghost[2 * d + 1];
    npt *= (size_t)ext[d];
  }
  const size_t es = precision == PMGPU_FP64 ? 8 : 4;
  std::vector<unsigned char> host;
  const unsigned char *src = static_cast<const unsigned char *>(mesh);
  if (device) {
    host.resize(es * 3 * npt);
    if (cudaMemcpy(host.data(), mesh, host.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      set_error(caller, "could not copy the mesh from the device.");
      return -1;
    }
    src = host.data();
  }
  out.clear();
  out.reserve((size_t)3 * t->ncell[0] * t->ncell[1] * t->ncell[2]);
  for (int k = 0; k < t->ncell[2]; k++)
    for (int j = 0; j < t->ncell[1]; j++)
      for (int i = 0; i < t->ncell[0]; i++) {
        const size_t q = (((size_t)(k + t->nghost[4]) * ext[1] + (j + t->nghost[2])) * ext[0] + (i + t->nghost[0])) * 3;
        for (int c = 0; c < 3; c++)
          out.push_back(precision == PMGPU_FP64 ? (float)reinterpret_cast<const double *>(src)[q + c]
                                                : reinterpret_cast<const float *>(src)[q + c]);
      }
  return 0;
}

}  // namespace

int pmgpu_output_pvti(const char *path, const char *tag, const pmgpu_patch *patch, int npieces, const int *icell,
                      const int *ncell) {
  const char *caller = "pmlib_output_mesh";
  if (!path || !tag || !patch || npieces < 1 || !icell || !ncell) {
    set_error(caller, "missing argument.");
    return -1;
  }
  FILE *f = fopen(path, "w");
  if (!f) {
    set_error(caller, "could not open the .pvti file.");
    return -1;
  }
  const int whole0[3] = {1, 1, 1};
  std::string s = "<?xml version=\"1.0\"?>\n";
  s += "<VTKFile type=\"PImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  s += "  <PImageData WholeExtent=\"" + extent6(whole0, patch->ncell) + origin_spacing(patch) + "\n";
  s += "    <PCellData Vectors=\"output\">\n";
  s += "      <PDataArray type=\"Float32\" Name=\"vort\" NumberOfComponents=\"3\" format=\"appended\" offset=\"0\"/>\n";
  s += "      <PDataArray type=\"Float32\" Name=\"vel\" NumberOfComponents=\"3\" format=\"appended\" offset=\"0\"/>\n";
  s += "    </PCellData>\n";
  for (int p = 0; p < npieces; p++) {
    char src[64];
    snprintf(src, sizeof(src), "_P%05d.vti", p);
    s += "    <Piece  Extent=\"" + extent6(icell + 3 * p, ncell + 3 * p) + "\" Source=\"" + tag + src + "\"/>\n";
  }
  s += "  </PImageData>\n</VTKFile>\n";
  const bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
  if (fclose(f) != 0 || !ok) {
    set_error(caller, "could not write the .pvti file.");
    return -1;
  }
  return 0;
}

int pmgpu_output_mesh(const char *outdir, const char *tag, const pmgpu_patch *patch, const pmgpu_topo *topo,
                      int precision, const void *mesh_vort, const void *mesh_vel, int device) {
  const char *caller = "pmlib_output_mesh";
  if (!outdir || !tag || !patch || !topo || !mesh_vort || !mesh_vel ||
      (precision != PMGPU_FP64 && precision != PMGPU_FP32)) {
    set_error(caller, "missing argument.");
    return -1;
  }
  const int icell[3] = {1, 1, 1};  // one rank: the cuboid starts at the patch's first cell
  const std::string base = std::string(outdir) + tag;
  if (pmgpu_output_pvti((base + ".pvti").c_str(), tag, patch, 1, icell, topo->ncell)) return -1;
  std::vector<float> w, u;
  if (interior_f32(topo, precision, mesh_vort, device, w, caller) ||
      interior_f32(topo, precision, mesh_vel, device, u, caller))
    return -1;
  FILE *f = fopen((base + "_P00000.vti").c_str(), "wb");
  if (!f) {
    set_error(caller, "could not open the .vti file.");
    return -1;
  }
  const long long ndata = (long long)topo->ncell[0] * topo->ncell[1] * topo->ncell[2];
  const int nb = (int)(3 * ndata * 4);
  std::string s = "<?xml version=\"1.0\"?>";
  s += "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">";
  s += "  <ImageData WholeExtent=\"" + extent6(icell, topo->ncell) + origin_spacing(patch);
  s += "<Piece Extent=\"" + extent6(icell, topo->ncell) + "\">";
  s += "<PointData></PointData><CellData>";
  s += "<DataArray type=\"Float32\" Name=\"vort\" NumberOfComponents=\"3\" format=\"appended\" offset=\"" +
       fmt_i(0, 10) + "\"/>";
  s += "<DataArray type=\"Float32\" Name=\"vel\" NumberOfComponents=\"3\" format=\"appended\" offset=\"" +
       fmt_i((long long)nb + 4, 10) + "\"/>";
  s += "</CellData></Piece></ImageData><AppendedData encoding=\"raw\">_";
  bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
  ok = ok && fwrite(&nb, 4, 1, f) == 1 && fwrite(w.data(), 4, w.size(), f) == w.size();
  ok = ok && fwrite(&nb, 4, 1, f) == 1 && fwrite(u.data(), 4, u.size(), f) == u.size();
  const std::string tail = "</AppendedData></VTKFile>";
  ok = ok && fwrite(tail.data(), 1, tail.size(), f) == tail.size();
  if (fclose(f) != 0 || !ok) {
    set_error(caller, "could not write the .vti file.");
    return -1;
  }
  return 0;
}

int pmgpu_output_topology(const char *tag, const pmgpu_patch *patch, int ptype, const pmgpu_topo *topo) {
  const char *caller = "pmlib_output_topology";
  if (!tag || !patch || !topo) {
    set_error(caller, "missing argument.");
    return -1;
  }
  FILE *f = fopen((std::string(tag) + ".dat").c_str(), "w");
  if (!f) {
    set_error(caller, "could not open the topology file.");
    return -1;
  }
  auto F82 = [](double v) {  // Fortran F8.2
    char b[32];
    snprintf(b, sizeof(b), "%8.2f", v);
    return std::string(b);
  };
  const std::string bar = "#===========================================================================\n";
  const std::string dash = "#---------------------------------------------------------------------------\n";
  std::string s = bar + "## Topology\n" + bar + "\n";
  s += "# Patch type:             " + fmt_i(ptype, 2) + "\n";
  s += "# Minimum extend:         ";
  for (int d = 0; d < 3; d++) s += F82(patch->xmin[d]);
  s += "\n# Maximum extend:         ";
  for (int d = 0; d < 3; d++) s += F82(patch->xmax[d]);
  s += "\n# Resolution:                1/" + fmt_i(lround(1.0 / patch->dx[0]), 4) + "\n";
  s += "# Number of mesh cells:   ";
  for (int d = 0; d < 3; d++) s += fmt_i(patch->ncell[d], 8);
  s += "\n# FFT-seq:                ";
  for (int d = 0; d < 3; d++) s += fmt_i(patch->fft_seq[d], 2);
  s += "\n\n" + dash + "# Topology for processor: " + fmt_i(0, 4) + "\n" + dash + "\n";
  s += "#  Number of particles:    " + fmt_i(topo->npart, 8) + "\n";
  s += "#  Minimum extend:         ";
  for (int d = 0; d < 3; d++) s += F82(topo->xmin[d]);
  s += "\n#  Maximum extend:         ";
  for (int d = 0; d < 3; d++) s += F82(topo->xmax[d]);
  s += "\n#  Number of mesh cells:   ";
  for (int d = 0; d < 3; d++) s += fmt_i(topo->ncell[d], 8);
  s += "\n#  Number of ghost cells:  ";
  for (int d = 0; d < 6; d++) s += fmt_i(topo->nghost[d], 4);
  s += "\n#  Boundary conditions:    ";
  for (int d = 0; d < 6; d++) s += fmt_i(topo->bound_cond[d], 4);
  s += "\n#  Neighbours:             ";
  // one rank: a periodic face's neighbour is the rank itself, a free face has none
  for (int d = 0; d < 6; d++) s += fmt_i(topo->bound_cond[d] != 0 ? 0 : -1, 4);
  s += "\n\n";
  const bool ok = fwrite(s.data(), 1, s.size(), f) == s.size();
  if (fclose(f) != 0 || !ok) {
    set_error(caller, "could not write the topology file.");
    return -1;
  }
  return 0;
}

namespace {
bool put_record(FILE *f, const void *p, int n) {
  return fwrite(&n, 4, 1, f) == 1 && fwrite(p, 1, (size_t)n, f) == (size_t)n && fwrite(&n, 4, 1, f) == 1;
}
bool get_record(FILE *f, void *p, int n) {
  int a = 0, b = 0;
  if (fread(&a, 4, 1, f) != 1 || a != n) return false;
  if (fread(p, 1, (size_t)n, f) != (size_t)n) return false;
  return fread(&b, 4, 1, f) == 1 && b == n;
}
}  // namespace

int pmgpu_output_particles(const char *tag, int itime_next, double time_next, int precision, int npart,
                           const void *pos, const void *vort, int device) {
  const char *caller = "pmlib_output_particle";
  if (!tag || npart < 0 || (npart > 0 && (!pos || !vort)) || (precision != PMGPU_FP64 && precision != PMGPU_FP32)) {
    set_error(caller, "missing argument.");
    return -1;
  }
  const size_t es = precision == PMGPU_FP64 ? 8 : 4, nb = es * 3 * (size_t)npart;
  std::vector<unsigned char> hp, hv;
  const unsigned char *p = static_cast<const unsigned char *>(pos), *v = static_cast<const unsigned char *>(vort);
  if (device && npart > 0) {
    hp.resize(nb);
    hv.resize(nb);
    if (cudaMemcpy(hp.data(), pos, nb, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hv.data(), vort, nb, cudaMemcpyDeviceToHost) != cudaSuccess) {
      set_error(caller, "could not copy the particles from the device.");
      return -1;
    }
    p = hp.data();
    v = hv.data();
  }
  FILE *f = fopen((std::string(tag) + ".dat").c_str(), "wb");
  if (!f) {
    set_error(caller, "could not open the particle file.");
    return -1;
  }
  bool ok = put_record(f, &itime_next, 4);
  if (precision == PMGPU_FP64) ok = ok && put_record(f, &time_next, 8);
  else {
    const float t = (float)time_next;
    ok = ok && put_record(f, &t, 4);
  }
  ok = ok && put_record(f, &npart, 4);
  unsigned char rec[48];
  for (int j = 0; ok && j < npart; j++) {  // one record (pos, vort) per particle
    memcpy(rec, p + es * 3 * j, es * 3);
    memcpy(rec + es * 3, v + es * 3 * j, es * 3);
    ok = put_record(f, rec, (int)(6 * es));
  }
  if (fclose(f) != 0 || !ok) {
    set_error(caller, "could not write the particle file.");
    return -1;
  }
  printf("[%04d](%s) : %s\n", 0, caller, "Saved particles.");
  fflush(stdout);
  return 0;
}

int pmgpu_input_particles(const char *file, double trunc, int precision, int max_part, void *pos, void *vort,
                          int *npart, int *itime, double *time) {
  const char *caller = "input_particles";
  if (!file || !npart || (precision != PMGPU_FP64 && precision != PMGPU_FP32)) {
    set_error(caller, "missing argument.");
    return -1;
  }
  FILE *f = fopen(file, "rb");
  if (!f) {
    set_error(caller, "could not open the particle file.");
    return -1;
  }
  const size_t es = precision == PMGPU_FP64 ? 8 : 4;
  int it = 0, nglob = 0;
  double tm = 0.0;
  bool ok = get_record(f, &it, 4);
  if (precision == PMGPU_FP64) ok = ok && get_record(f, &tm, 8);
  else {
    float t = 0.f;
    ok = ok && get_record(f, &t, 4);
    tm = t;
  }
  ok = ok && get_record(f, &nglob, 4);
  int kept = 0;
  unsigned char rec[48];
  for (int i = 0; ok && i < nglob; i++) {
    ok = get_record(f, rec, (int)(6 * es));
    if (!ok) break;
    double w[3];
    for (int c = 0; c < 3; c++)
      w[c] = es == 8 ? reinterpret_cast<const double *>(rec)[3 + c] : reinterpret_cast<const float *>(rec)[3 + c];
    if (std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) >= trunc) {  // input_particles.f:83-86
      if (kept < max_part && pos && vort) {
        memcpy(static_cast<unsigned char *>(pos) + es * 3 * kept, rec, es * 3);
        memcpy(static_cast<unsigned char *>(vort) + es * 3 * kept, rec + es * 3, es * 3);
      }
      kept++;
    }
  }
  fclose(f);
  if (!ok) {
    set_error(caller, "the particle file is not a restart file of this precision.");
    return -1;
  }
  if (kept == 0) {
    set_error(caller, "No particles above truncation value.");
    return -1;
  }
  *npart = kept;
  if (itime) *itime = it;
  if (time) *time = tm;
  if (kept > max_part && (pos || vort)) {
    set_error(caller, "more particles above the truncation value than max_part.");
    return -1;
  }
  return 0;
}
