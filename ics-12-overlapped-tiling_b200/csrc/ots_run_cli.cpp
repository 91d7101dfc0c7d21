// ots_run_cli.cpp -- drop-in for the reference runners build.out/ocl-<stencil>.
//
// One binary for all thirteen stencils: the stencil comes from the program
// name (ots-jacobi-2d, ... as symlinks to ots-run) or from --stencil.  The
// flags and their defaults are the reference's
// (opencl/jacobi-2d/jacobi-2d.cpp:566-607, opencl/jacobi-3d/jacobi-3d.cpp:486-523,
// opencl/jacobi-1d/jacobi-1d.cpp:404-438) and the output is its "Key: value"
// protocol (opencl/common/inc/CLCommon.hpp:23-27), which
// scripts/utils.py:104-156 and scripts/results-to-csv.py parse.  The work
// itself goes through libots (include/ots.h).
//
// -v/--verify runs the runner's own naive CPU sweep and prints
// "Error Norm", "Ref Norm" and "Correctness" exactly as compareResults
// (opencl/jacobi-2d/jacobi-2d.cpp:517-551) does.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ots.h"
#include "ots_ops.cuh"

namespace {

void usage(const char* prog) {
  fprintf(stderr,
          "Usage: %s [options]\n"
          "  -h, --help                   Show usage information\n"
          "  -n, --problem-size N         Set problem size\n"
          "  -t, --time-steps N           Set number of time steps\n"
          "  -x, --block-size-x N         Set block size (X)\n"
          "  -y, --block-size-y N         Set block size (Y)\n"
          "  -z, --block-size-z N         Set block size (Z)\n"
          "  -e, --elements-per-thread N  Set elements per thread\n"
          "  -s, --time-tile-size N       Set time tile size\n"
          "  -p, --phase-limit N          Stop after a certain kernel phase (1, 2, 3)\n"
          "  -f, --load-kernel FILE       (rejected: kernels are compiled ahead of time)\n"
          "  -w, --save-kernel FILE       Save a description of the chosen kernel\n"
          "  -v, --verify                 Verify results against a CPU sweep\n"
          "  -c, --dump-clocks BOOL       Dump per-warp phase clocks (tile kernel) to stderr\n"
          "  -b, --break-threads          Accepted for compatibility\n"
          "      --time-only WHAT         Accepted for compatibility (gmem, instr, smem)\n"
          "      --stencil NAME           Stencil (default: from the program name)\n"
          "      --engine compat|native   Geometry derivation (default compat)\n"
          "      --kernel auto|tile|stream|plain|tex\n"
          "      --variant ref|baseline|fast  Arithmetic variant (default: ref for compat;\n"
          "                               fast: approximate division, rician / tv / cs-3d)\n"
          "      --stream-impl N          Stream kernels' arithmetic: 0 packed FP32 where it\n"
          "                               applies (default), 1 scalar\n"
          "      --coef X                 Averaging weight (Jacobi stencils)\n"
          "      --seed N                 srand seed for the input fill (default 123456)\n"
          "      --init ref|baseline      Inputs: the reference fill everywhere (default), or the\n"
          "                               benchmark workloads' (Poisson f = 2u - 1; Rician / TV:\n"
          "                               disk image with Rician noise, u0 = F = f, V = 1)\n"
          "      --plain                  Also time the plain one-step kernel\n"
          "      --device N               CUDA device\n",
          prog);
}

struct Acc {
  const float* const* f;
  int64_t i;
  int64_t sy, sz;
  int x, y, z;  // padded coordinates
  int lo, hi, dims;
  bool in(int xx, int yy, int zz) const {
    if (xx < lo || xx >= hi) return false;
    if (dims >= 2 && (yy < lo || yy >= hi)) return false;
    if (dims >= 3 && (zz < lo || zz >= hi)) return false;
    return true;
  }
  float operator()(int fi, int dz, int dy, int dx) const {
    return in(x + dx, y + dy, z + dz) ? f[fi][i + dz * sz + dy * sy + dx] : 0.0f;
  }
  bool inside(int dz, int dy, int dx) const { return in(x + dx, y + dy, z + dz); }
  int gy() const { return y - lo; }
};

template <class Op>
void cpu_sweep(std::vector<std::vector<float>>& st, const std::vector<std::vector<float>>& aux,
               int dims, int P, int lo, int hi, int steps, const ots::OpArgs& op) {
  const int64_t sy = P, sz = (int64_t)P * P;
  std::vector<std::vector<float>> nb = st;
  const int zlo = dims == 3 ? lo : 0, zhi = dims == 3 ? hi : 1;
  const int ylo = dims >= 2 ? lo : 0, yhi = dims >= 2 ? hi : 1;
  std::vector<const float*> fp(st.size());
  for (int t = 0; t < steps; ++t) {
    for (size_t f = 0; f < st.size(); ++f) fp[f] = st[f].data();
    for (int z = zlo; z < zhi; ++z)
      for (int y = ylo; y < yhi; ++y)
        for (int x = lo; x < hi; ++x) {
          const int64_t i = (dims == 3 ? z * sz : 0) + (dims >= 2 ? y * sy : 0) + x;
          Acc a{fp.data(), i, sy, sz, x, y, z, lo, hi, dims};
          float av[2] = {0.0f, 0.0f};
          for (size_t k = 0; k < aux.size(); ++k) av[k] = aux[k][i];
          float res[3];
          Op::apply(a, av, op, t, res);
          for (size_t f = 0; f < st.size(); ++f) nb[f][i] = res[f];
        }
    std::swap(st, nb);
  }
}

void cpu_reference(int stencil, std::vector<std::vector<float>>& st,
                   const std::vector<std::vector<float>>& aux, int dims, int P, int lo, int hi,
                   int steps, const ots::OpArgs& op) {
  using namespace ots;
  switch (stencil) {
    case OTS_JACOBI_1D: cpu_sweep<OpJacobi1D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_JACOBI_1D_5PT: cpu_sweep<OpJacobi1D5>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_JACOBI_1D_7PT: cpu_sweep<OpJacobi1D7>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_JACOBI_2D: cpu_sweep<OpJacobi2D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_JACOBI_3D: cpu_sweep<OpJacobi3D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_POISSON_2D: cpu_sweep<OpPoisson2D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_POISSON_3D: cpu_sweep<OpPoisson3D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_GRADIENT_2D: cpu_sweep<OpGradient2D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_GRADIENT_3D: cpu_sweep<OpGradient3D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_FDTD_2D: cpu_sweep<OpFdtd2D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_RICIAN_DENOISE_2D: cpu_sweep<OpRician2D>(st, aux, dims, P, lo, hi, steps, op); break;
    case OTS_CDSC_TV_UPDATE_2D: cpu_sweep<OpTvUpdate2D>(st, aux, dims, P, lo, hi, steps, op); break;
    default: cpu_sweep<OpCs3D>(st, aux, dims, P, lo, hi, steps, op); break;
  }
}

void print_kv(const char* key, const char* value, void*) { printf("%s: %s\n", key, value); }

bool parse_bool(const char* s) {
  return !(strcmp(s, "0") == 0 || strcmp(s, "false") == 0 || strcmp(s, "no") == 0);
}

}  // namespace

int main(int argc, char** argv) {
  std::string prog = argv[0];
  const size_t slash = prog.find_last_of('/');
  const std::string base = slash == std::string::npos ? prog : prog.substr(slash + 1);
  int stencil = -1;
  if (base.rfind("ots-", 0) == 0) stencil = ots_stencil_from_name(base.c_str() + 4);

  ots_params p;
  memset(&p, 0, sizeof p);
  p.problem_size = -1;
  p.time_steps = 64;
  p.block_x = 16;
  p.block_y = 16;
  p.block_z = -1;
  p.elements_per_thread = 1;
  p.time_tile = 1;
  p.engine = OTS_ENGINE_COMPAT;
  p.kernel = OTS_KERNEL_AUTO;
  p.variant = -1;
  unsigned seed = 123456;  // srand(123456), opencl/jacobi-2d/jacobi-2d.cpp:561
  bool verify = false, plain = false, bx_set = false, by_set = false, dump_clocks = false;
  bool init_baseline = false;
  std::string save_kernel, load_kernel;

  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    std::string val;
    const size_t eq = a.find('=');
    if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
      val = a.substr(eq + 1);
      a = a.substr(0, eq);
    }
    auto next = [&]() -> const char* {
      if (!val.empty()) return val.c_str();
      if (i + 1 >= argc) {
        fprintf(stderr, "ERROR: option %s needs a value\n", a.c_str());
        exit(1);
      }
      return argv[++i];
    };
    if (a == "-h" || a == "--help") {
      usage(argv[0]);
      return 1;
    } else if (a == "-n" || a == "--problem-size") p.problem_size = atoi(next());
    else if (a == "-t" || a == "--time-steps") p.time_steps = atoi(next());
    else if (a == "-x" || a == "--block-size-x") {
      p.block_x = atoi(next());
      bx_set = true;
    } else if (a == "-y" || a == "--block-size-y") {
      p.block_y = atoi(next());
      by_set = true;
    }
    else if (a == "-z" || a == "--block-size-z") p.block_z = atoi(next());
    else if (a == "-e" || a == "--elements-per-thread") p.elements_per_thread = atoi(next());
    else if (a == "-s" || a == "--time-tile-size") p.time_tile = atoi(next());
    else if (a == "-p" || a == "--phase-limit") p.phase_limit = atoi(next());
    else if (a == "-f" || a == "--load-kernel") load_kernel = next();
    else if (a == "-w" || a == "--save-kernel") save_kernel = next();
    else if (a == "-v" || a == "--verify") verify = true;
    else if (a == "-c" || a == "--dump-clocks") dump_clocks = parse_bool(next());
    else if (a == "-b" || a == "--break-threads") {
    } else if (a == "--time-only") (void)next();
    else if (a == "--stencil") stencil = ots_stencil_from_name(next());
    else if (a == "--engine") p.engine = strcmp(next(), "native") == 0 ? OTS_ENGINE_NATIVE : OTS_ENGINE_COMPAT;
    else if (a == "--kernel") {
      const std::string k = next();
      p.kernel = k == "tile" ? OTS_KERNEL_TILE : k == "stream" ? OTS_KERNEL_STREAM
                 : k == "plain" ? OTS_KERNEL_PLAIN : k == "tex" ? OTS_KERNEL_TEX : OTS_KERNEL_AUTO;
    } else if (a == "--variant") {
      const char* v = next();
      p.variant = strcmp(v, "baseline") == 0 ? OTS_VARIANT_BASELINE
                  : strcmp(v, "fast") == 0   ? OTS_VARIANT_FAST
                                             : OTS_VARIANT_REF;
    } else if (a == "--stream-impl") p.stream_impl = atoi(next());
    else if (a == "--coef") p.coef = (float)atof(next());
    else if (a == "--seed") seed = (unsigned)strtoul(next(), nullptr, 10);
    else if (a == "--init") init_baseline = strcmp(next(), "baseline") == 0;
    else if (a == "--plain") plain = true;
    else if (a == "--device") p.device = atoi(next());
    else {
      fprintf(stderr, "ERROR: unknown option %s\n", a.c_str());
      usage(argv[0]);
      return 1;
    }
  }
  if (stencil < 0) {
    fprintf(stderr, "ERROR: no stencil (use --stencil NAME or run as ots-<stencil>)\n");
    return 1;
  }
  if (!load_kernel.empty()) {
    printf("ERROR: --load-kernel is not supported: kernels are compiled ahead of time\n");
    return 1;
  }
  p.stencil = stencil;
  const int dims = ots_stencil_dims(stencil);
  if (p.problem_size < 0) p.problem_size = dims == 3 ? 128 : (dims == 1 ? 1024 : 1024);
  if (p.block_z < 0) p.block_z = dims == 3 ? 8 : 1;
  if (dims == 3) {
    // 3D runner defaults, opencl/jacobi-3d/jacobi-3d.cpp:486-523
    if (!bx_set) p.block_x = 8;
    if (!by_set) p.block_y = 8;
  }
  if (dims == 1) p.block_y = p.block_z = 1;
  if (dims == 2) p.block_z = 1;
  if (p.variant < 0) p.variant = p.engine == OTS_ENGINE_COMPAT ? OTS_VARIANT_REF : OTS_VARIANT_BASELINE;

  ots_plan* plan = nullptr;
  ots_status st = ots_plan_create(&p, &plan);
  if (st != OTS_OK) {
    printf("ERROR: %s\n", ots_last_error());
    return 1;
  }
  ots_geometry g;
  ots_plan_geometry(plan, &g);
  ots_describe(plan, print_kv, nullptr);
  char devname[256] = {0};
  int32_t sms = 0;
  ots_device_info(p.device, devname, sizeof devname, &sms, nullptr, nullptr);
  printf("Device: %s\n", devname);

  if (!save_kernel.empty()) {
    FILE* fh = fopen(save_kernel.c_str(), "w");
    if (fh) {
      static const char* kn[] = {"auto", "tile", "stream", "plain"};
      fprintf(fh, "/* ots kernel instantiation (compiled ahead of time for sm_100a) */\n");
      fprintf(fh, "stencil=%s kernel=%s E=%d T=%d threads=%dx%dx%d e_axis=%d smem=%lld regs=%d\n",
              ots_stencil_name(stencil), kn[g.kernel & 3], p.elements_per_thread, p.time_tile,
              g.threads[0], g.threads[1], g.threads[2], g.e_axis, (long long)g.shared_bytes,
              g.registers);
      fclose(fh);
    }
  }

  // Host arrays in the reference layout, filled as the reference does.
  const int P = g.padded_size, lo = g.padding, hi = g.padding + g.real_size;
  int64_t cells = 1;
  for (int d = 0; d < dims; ++d) cells *= P;
  const int ns = g.num_fields, na = g.num_aux;
  std::vector<std::vector<float>> state(ns, std::vector<float>(cells)), aux(na, std::vector<float>(cells));
  std::vector<float*> fillp;
  for (auto& v : state) fillp.push_back(v.data());
  for (auto& v : aux) fillp.push_back(v.data());
  ots_fill_reference(dims, P, g.padding, g.real_size, seed, fillp.data(), ns + na);
  if (init_baseline && (stencil == OTS_POISSON_2D || stencil == OTS_POISSON_3D)) {
    for (float& f : aux[0]) f = f != 0.0f ? 2.0f * f - 1.0f : 0.0f;  // f uniform [-1, 1)
  } else if (init_baseline &&
             (stencil == OTS_RICIAN_DENOISE_2D || stencil == OTS_CDSC_TV_UPDATE_2D)) {
    const int n = g.real_size;
    std::vector<float> img((size_t)n * n);
    ots_fill_disks(n, 2012, 64, 0.1f, 0.05f, img.data(), nullptr);
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const size_t i = (size_t)(y + lo) * P + (x + lo), j = (size_t)y * n + x;
        state[0][i] = aux[0][i] = img[j];
        if (na > 1) aux[1][i] = 1.0f;  // V
      }
  }

  std::vector<std::vector<float>> ref;
  if (verify) {
    ref = state;
    ots::OpArgs op{g.coef, g.h2, p.variant};
    cpu_reference(stencil, ref, aux, dims, P, lo, hi, p.time_steps, op);
  }

  std::vector<const float*> sp, ap;
  for (auto& v : state) sp.push_back(v.data());
  for (auto& v : aux) ap.push_back(v.data());
  st = ots_upload(plan, sp.data(), ap.empty() ? nullptr : ap.data());
  if (st == OTS_OK && dump_clocks && ots_plan_enable_clocks(plan, 1) != OTS_OK)
    fprintf(stderr, "warning: clock dump unavailable: %s\n", ots_last_error());
  ots_timing tm{};
  if (st == OTS_OK) st = ots_run(plan, OTS_KERNEL_AUTO, &tm);
  if (st == OTS_OK && dump_clocks) {
    // opencl/jacobi-2d/jacobi-2d.cpp:957-996: the warps that ran on SM 1
    int64_t n = 0;
    if (ots_plan_clock_records(plan, nullptr, 0, &n) == OTS_OK && n > 0) {
      std::vector<ots_clock_record> recs((size_t)n);
      if (ots_plan_clock_records(plan, recs.data(), n, &n) == OTS_OK) {
        fprintf(stderr, "bx,by,warp,sm,clock0,clock1,clock2,clock3,clock4,\n");
        for (const ots_clock_record& r : recs)
          if (r.sm == 1)
            fprintf(stderr, "%u,%u,%u,%u,%u,%u,%u,%u,%u,\n", r.block_x,
                    r.block_y + r.block_z * (uint32_t)g.num_blocks[1], r.warp, r.sm, r.clock[0],
                    r.clock[1], r.clock[2], r.clock[3], r.clock[4]);
      }
    }
  }
  std::vector<float*> dp;
  for (auto& v : state) dp.push_back(v.data());
  if (st == OTS_OK) st = ots_download(plan, dp.data());
  if (st != OTS_OK) {
    printf("ERROR: %s\n", ots_last_error());
    ots_plan_destroy(plan);
    return 1;
  }
  const double ev_s = tm.event_ms * 1e-3;
  printf("EventElapsed: %.9g\n", ev_s);
  printf("ProfileTimerResolution: %d\n", 500);
  printf("Elapsed Time: %.9g\n", tm.wall_s);
  const double upd = (double)g.interior_points * p.time_steps;
  printf("Actual GFlop/s: %.9g\n", upd * g.flops_per_point / tm.wall_s / 1e9);
  printf("Real Size: %d\n", g.real_size);
  double dev_pts = (double)g.threads[0] * g.threads[1] * g.threads[2] * p.elements_per_thread *
                   g.num_blocks[0] * g.num_blocks[1] * g.num_blocks[2];
  printf("Device GFlop/s: %.9g\n", dev_pts * g.flops_per_point * p.time_steps / tm.wall_s / 1e9);
  printf("GUpdates/s: %.9g\n", ev_s > 0 ? upd / ev_s / 1e9 : 0.0);
  printf("Launches: %d\n", tm.launches);

  if (plain) {
    st = ots_upload(plan, sp.data(), ap.empty() ? nullptr : ap.data());
    ots_timing tp{};
    if (st == OTS_OK) st = ots_run(plan, OTS_KERNEL_PLAIN, &tp);
    if (st == OTS_OK)
      printf("Plain GUpdates/s: %.9g\n", upd / (tp.event_ms * 1e-3) / 1e9);
    else
      printf("Plain GUpdates/s: ERROR %s\n", ots_last_error());
  }

  if (verify) {
    // compareResults, opencl/jacobi-2d/jacobi-2d.cpp:517-551 (field 0)
    double e = 0.0, r = 0.0;
    const int zlo = dims == 3 ? lo : 0, zhi = dims == 3 ? hi : 1;
    const int ylo = dims >= 2 ? lo : 0, yhi = dims >= 2 ? hi : 1;
    for (int z = zlo; z < zhi; ++z)
      for (int y = ylo; y < yhi; ++y)
        for (int x = lo; x < hi; ++x) {
          const int64_t i = (dims == 3 ? (int64_t)z * P * P : 0) + (dims >= 2 ? (int64_t)y * P : 0) + x;
          const float h = ref[0][i], d = state[0][i];
          const double diff = h - d;
          e += diff * diff;
          r += h * h;
        }
    e = std::sqrt(e);
    r = std::sqrt(r);
    printf("Error Norm: %.9g\n", e);
    printf("Ref Norm: %.9g\n", r);
    const bool pass = !(std::fabs(r) < 1e-7) && !(e / r > 1e-2);
    printf("Correctness: %s\n", pass ? "PASSED" : "FAILED");
  }
  ots_plan_destroy(plan);
  return 0;
}
