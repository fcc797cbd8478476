// Drives the C++ TaskManager layer (include/tmx_taskmanager.hpp) the way
// CosTuuM's Python module drives its TaskManager in get_table
// (src/CTMModule.cpp:146-478): construct the distributions and the
// TaskManager, add the grid, generate_tasks, QuickSched::execute_tasks, then
// read every coefficient through the ResultKey and the result objects into
// arrays [type][size][wavelength][theta][k] (k = Qabs, Qabspol, then Qext,
// Qextpol, Qextcpol) and [type][size][wavelength][theta][phi][4][4].
//
// Cases: the grids of the golden get_table fixtures (tests/golden/
// tables.npz, made by the unmodified reference). Each array is written as
// raw little-endian doubles to <outdir>/<name>.bin.
//
// Usage: drive_get_table <outdir>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "tmx_taskmanager.hpp"

using namespace tmx;

namespace {

struct Table {
  std::vector<double> q, z;
};

// the body of get_table after argument parsing
Table get_table(const std::vector<int_fast32_t> &types,
                const std::vector<double> &sizes,
                const std::vector<double> &wavelengths,
                const std::vector<double> &thetas, const ShapeDistribution &shape,
                const AlignmentDistribution &align, const DustProperties &dust,
                uint_fast32_t nmin, uint_fast32_t nmax, uint_fast32_t glfac,
                double tolerance, uint_fast32_t ngauss, bool do_absorption,
                bool do_extinction, bool do_scattering,
                bool account_for_scattering) {
  TaskManager task_manager(nmin, nmax, glfac, tolerance, (size_t)1e10, shape,
                           align, dust);
  for (auto t : types) {
    task_manager.add_composition(t);
  }
  for (double s : sizes) {
    task_manager.add_size(s);
  }
  for (double w : wavelengths) {
    task_manager.add_wavelength(w);
  }
  QuickSched quicksched(4, false, "", false);
  std::vector<Task *> tasks;
  std::vector<Resource *> resources;
  ResultKey *result_key = nullptr;
  std::vector<Result *> results;
  TMatrixAuxiliarySpaceManager *space_manager = nullptr;
  task_manager.generate_tasks(thetas, ngauss, quicksched, tasks, resources,
                              result_key, results, space_manager, do_extinction,
                              do_absorption, do_scattering,
                              account_for_scattering, false, false, "");
  quicksched.execute_tasks();
  for (Task *t : tasks) {
    delete t;
  }
  for (Resource *r : resources) {
    delete r;
  }
  delete space_manager;

  Table out;
  const size_t nt = result_key->composition_size();
  const size_t ns = result_key->size_size();
  const size_t nl = result_key->wavelength_size();
  const size_t nth = thetas.size();
  if (do_absorption || do_extinction) {
    const size_t nk = (do_absorption ? 2 : 0) + (do_extinction ? 3 : 0);
    out.q.assign(nt * ns * nl * nth * nk, 0.);
    for (size_t it = 0; it < nt; ++it) {
      for (size_t is = 0; is < ns; ++is) {
        for (size_t il = 0; il < nl; ++il) {
          for (size_t ith = 0; ith < nth; ++ith) {
            double *dst = out.q.data() + (((it * ns + is) * nl + il) * nth + ith) * nk;
            size_t k = 0;
            if (do_absorption) {
              const auto &r = *static_cast<AbsorptionCoefficientResult *>(
                  results[result_key->get_result_index(it, is, il, do_extinction)]);
              dst[k++] = r.get_Qabs(ith);
              dst[k++] = r.get_Qabspol(ith);
            }
            if (do_extinction) {
              const auto &r = *static_cast<ExtinctionCoefficientResult *>(
                  results[result_key->get_result_index(it, is, il, 0)]);
              dst[k++] = r.get_Qext(ith);
              dst[k++] = r.get_Qextpol(ith);
              dst[k++] = r.get_Qextcpol(ith);
            }
          }
        }
      }
    }
  }
  if (do_scattering) {
    const uint_fast32_t idx = (do_extinction ? 1 : 0) + (do_absorption ? 1 : 0);
    out.z.assign(nt * ns * nl * nth * 2 * nth * 16, 0.);
    for (size_t it = 0; it < nt; ++it) {
      for (size_t is = 0; is < ns; ++is) {
        for (size_t il = 0; il < nl; ++il) {
          const auto &r = *static_cast<ScatteringMatrixResult *>(
              results[result_key->get_result_index(it, is, il, idx)]);
          for (size_t ith = 0; ith < nth; ++ith) {
            for (size_t iphi = 0; iphi < 2 * nth; ++iphi) {
              const auto &Z = r.get_scattering_matrix(2 * ith * nth + iphi);
              double *dst = out.z.data() +
                            ((((it * ns + is) * nl + il) * nth + ith) * 2 * nth + iphi) * 16;
              for (int row = 0; row < 4; ++row) {
                for (int col = 0; col < 4; ++col) {
                  dst[4 * row + col] = Z(row, col);
                }
              }
            }
          }
        }
      }
    }
  }
  delete result_key;
  for (Result *r : results) {
    delete r;
  }
  return out;
}

std::complex<double> m_const_15(double, double, int32_t, void *) {
  return {1.5, 0.02};
}
std::complex<double> m_grid(double w, double s, int32_t, void *) {
  return {1.4 + 0.3 * s / 1e-6, 0.05 * (1e-6 / w)};
}
std::complex<double> m_by_type(double, double, int32_t t, void *) {
  return {1.4 + 0.1 * t, 0.05};
}
std::complex<double> m_const_16(double, double, int32_t, void *) {
  return {1.6, 0.2};
}

bool write(const std::string &dir, const std::string &name,
           const std::vector<double> &v) {
  const std::string path = dir + "/" + name + ".bin";
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) {
    return false;
  }
  const bool ok = fwrite(v.data(), sizeof(double), v.size(), f) == v.size();
  return fclose(f) == 0 && ok;
}

} // namespace

int main(int argc, char **argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s <outdir>\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  try {
    // one grain, Q_ext / Q_abs at 32 zenith angles uniform in cos(theta)
    std::vector<double> th1(32);
    for (int i = 0; i < 32; ++i) {
      // numpy.linspace(-1, 1, 32): i * (2 / 31) - 1, the last point exactly 1
      th1[i] = std::acos(i == 31 ? 1. : i * (2. / 31.) + -1.);
    }
    {
      SingleShapeShapeDistribution shape(2.);
      SizeBasedAlignmentDistribution align(1e-5, 0, 40);
      CustomDustProperties dust(m_const_15);
      Table t = get_table({0}, {0.2e-6}, {1e-6}, th1, shape, align, dust, 10, 40,
                          2, 1e-4, 20, true, true, false, false);
      // (the angles too: the C library's acos and numpy's arccos may round
      // differently in the last bit)
      if (!write(dir, "gt1", t.q) || !write(dir, "gt1_theta", th1)) {
        return 1;
      }
    }
    // a small grid: Draine-Hensley shapes, Mishchenko alignment, scattering
    {
      DraineHensleyShapeDistribution shape(4);
      SizeBasedAlignmentDistribution align(0.1e-6, 1, 30);
      CustomDustProperties dust(m_grid);
      Table t = get_table({0}, {0.05e-6, 0.3e-6}, {1.5e-6, 0.8e-6}, {0.3, 1.2, 2.0},
                          shape, align, dust, 10, 30, 2, 1e-4, 20, true, true, true,
                          false);
      if (!write(dir, "gt2_q", t.q) || !write(dir, "gt2_z", t.z)) {
        return 1;
      }
    }
    // scattering subtraction, Davis-Greenstein alignment, two compositions
    {
      SingleShapeShapeDistribution shape(1.5);
      SizeBasedAlignmentDistribution align(1e-7, 0, 30);
      CustomDustProperties dust(m_by_type);
      Table t = get_table({0, 2}, {0.4e-6}, {1e-6, 2e-6}, {0.1, 1.0, 2.5}, shape,
                          align, dust, 10, 30, 2, 1e-4, 6, true, false, false, true);
      if (!write(dir, "gt3", t.q)) {
        return 1;
      }
    }
    // disabled alignment; custom (copied) oblate / prolate distributions
    {
      SingleShapeShapeDistribution shape(0.7);
      CustomDustProperties dust(m_const_16);
      SizeBasedAlignmentDistribution disabled(1e-7, 2, 30);
      Table t4 = get_table({0}, {0.3e-6}, {1e-6}, {0.5, 1.5}, shape, disabled, dust,
                           10, 30, 2, 1e-4, 20, true, true, false, false);
      MishchenkoOrientationDistribution ob(60, 0.7);
      DavisGreensteinOrientationDistribution pr(60, 0.5);
      SizeBasedAlignmentDistribution custom(1e-7, 3, 30, &ob, &pr);
      Table t5 = get_table({0}, {0.3e-6}, {1e-6}, {0.5, 1.5}, shape, custom, dust,
                           10, 30, 2, 1e-4, 20, true, true, false, false);
      if (!write(dir, "gt4", t4.q) || !write(dir, "gt5", t5.q)) {
        return 1;
      }
    }
  } catch (const std::exception &e) {
    fprintf(stderr, "drive_get_table: %s\n", e.what());
    return 1;
  }
  return 0;
}
