/* tmx_taskmanager.hpp -- C++ host layer with the shape of CosTuuM's
 * TaskManager, for callers that drive the T-matrix path from C++.
 *
 * CosTuuM's Python module builds its tables with (src/CTMModule.cpp:146-478)
 *
 *   TaskManager task_manager(nmin, nmax, glfac, tol, mem, shape, align, dust);
 *   task_manager.add_composition(..); add_size(..); add_wavelength(..);
 *   QuickSched quicksched(nthread, graph_log, graph_log_name, verbose);
 *   task_manager.generate_tasks(thetas, ngauss, quicksched, tasks, resources,
 *                               result_key, results, space_manager,
 *                               do_extinction, do_absorption, do_scattering,
 *                               account_for_scattering, verbose, ...);
 *   quicksched.execute_tasks();
 *   ... result_key->get_result_index(..) -> results[..]->get_Qabs(..) ...
 *
 * (TaskManager: src/TaskManager.hpp:371-455; QuickSched::execute_tasks:
 * src/QuickSchedWrapper.hpp:375; ResultKey: src/ResultKey.hpp; results:
 * src/AbsorptionCoefficientTask.hpp:40-110, ExtinctionCoefficientTask.hpp:
 * 40-125, ScatteringMatrixTask.hpp:40-100). The classes below keep those
 * names, constructors and accessors (namespace tmx), so such a driver
 * compiles against this header with `using namespace tmx;`. What changes
 * underneath: generate_tasks builds one device batch description instead of
 * a task graph (the task and resource lists stay empty), and the QuickSched
 * object is a handle that runs that batch on the GPU through tmx_get_table
 * (include/tmx.h) when execute_tasks() is called. The distributions are set
 * up by the library's host routines, bit-identical to the reference's
 * (tmx_shape_distribution, tmx_orientation_coefficients).
 *
 * Errors: the reference aborts through ctm_error; here a failed call throws
 * std::runtime_error with the library's message. Per-grain outcomes (not
 * converged, ...) are available from QuickSched::grain_status().
 *
 * Link with libtmx.so.
 */
#ifndef TMX_TASKMANAGER_HPP
#define TMX_TASKMANAGER_HPP

#include <algorithm>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "tmx.h"

namespace tmx {

typedef double float_type;

// ----------------------------------------------------------------- shapes --

/* Shape distribution: axis-ratio quadrature nodes and weights
 * (src/ShapeDistribution.hpp:95-137). The base class is the reference's
 * default distribution on [0.5, 1.5]. */
class ShapeDistribution {
protected:
  std::vector<float_type> _shapes, _weights;
  float_type _limits[2] = {0.5, 1.5};

  ShapeDistribution() {}
  void evaluate(int kind, uint_fast32_t npoints, double p1, double p2) {
    _shapes.assign(npoints, 0.);
    _weights.assign(npoints, 0.);
    if (tmx_shape_distribution(kind, (int)npoints, p1, p2, _shapes.data(),
                               _weights.data(), _limits) != TMX_OK) {
      throw std::runtime_error("tmx::ShapeDistribution: invalid arguments");
    }
  }

public:
  explicit ShapeDistribution(const uint_fast32_t npoints) {
    evaluate(0, npoints, 0., 0.);
  }
  virtual ~ShapeDistribution() {}
  virtual float_type get_minimum_axis_ratio() const { return _limits[0]; }
  virtual float_type get_maximum_axis_ratio() const { return _limits[1]; }
  uint_fast32_t get_number_of_points() const { return _shapes.size(); }
  float_type get_shape(const uint_fast32_t index) const { return _shapes.at(index); }
  float_type get_weight(const uint_fast32_t index) const { return _weights.at(index); }
};

/* Draine & Hensley (2017) CDE2 shape distribution
 * (src/DraineHensleyShapeDistribution.hpp:230). */
class DraineHensleyShapeDistribution : public ShapeDistribution {
public:
  DraineHensleyShapeDistribution(const uint_fast32_t npoints,
                                 const float_type cutoff = 0.15,
                                 const float_type fraction = -1.) {
    evaluate(1, npoints, cutoff, fraction);
  }
};

/* Every grain has the same axis ratio (src/SingleShapeShapeDistribution.hpp:
 * 70). */
class SingleShapeShapeDistribution : public ShapeDistribution {
public:
  explicit SingleShapeShapeDistribution(const float_type axis_ratio) {
    _shapes.assign(1, axis_ratio);
    _weights.assign(1, 1.);
    _limits[0] = _limits[1] = axis_ratio;
  }
};

// ------------------------------------------------------------ orientation --

/* Orientation distribution expansion coefficients p_0 .. p_nmax
 * (src/OrientationDistribution.hpp:192-270). The base class is random
 * orientation; initialise() computes its coefficients, as in the
 * reference. */
class OrientationDistribution {
protected:
  std::vector<float_type> _coefficients;

  void compute(int kind, double param, double (*fn)(double, void *), void *arg) {
    if (tmx_orientation_coefficients(kind, param,
                                     (int)_coefficients.size() - 1, fn, arg,
                                     _coefficients.data()) != TMX_OK) {
      throw std::runtime_error("tmx::OrientationDistribution: invalid arguments");
    }
  }

public:
  explicit OrientationDistribution(const uint_fast32_t nmax)
      : _coefficients(nmax + 1, 0.) {}
  virtual ~OrientationDistribution() {}
  void initialise() { compute(0, 0., nullptr, nullptr); }
  float_type get_coefficient(const uint_fast32_t n) const {
    return _coefficients.at(n);
  }
  uint_fast32_t get_maximum_order() const { return _coefficients.size() - 1; }
  virtual bool compute_alignment() const { return true; }
  const std::vector<float_type> &coefficients() const { return _coefficients; }
};

/* p(beta) = 1/2 + 5/4 p2 (3 cos^2 beta - 1)
 * (src/MishchenkoOrientationDistribution.hpp:105). */
class MishchenkoOrientationDistribution : public OrientationDistribution {
public:
  MishchenkoOrientationDistribution(const uint_fast32_t nmax,
                                    const float_type cos2beta)
      : OrientationDistribution(nmax) {
    compute(1, cos2beta, nullptr, nullptr);
  }
};

/* Perfect Davis-Greenstein alignment
 * (src/DavisGreensteinOrientationDistribution.hpp:76). */
class DavisGreensteinOrientationDistribution : public OrientationDistribution {
public:
  DavisGreensteinOrientationDistribution(const uint_fast32_t nmax,
                                         const float_type axis_ratio)
      : OrientationDistribution(nmax) {
    compute(2, axis_ratio, nullptr, nullptr);
  }
};

/* No orientation averaging at all
 * (src/DisabledAlignmentOrientationDistribution.hpp:70). */
class DisabledAlignmentOrientationDistribution : public OrientationDistribution {
public:
  DisabledAlignmentOrientationDistribution() : OrientationDistribution(0) {}
  bool compute_alignment() const override { return false; }
};

/* p(beta) from a callback fn(beta, arg) (the C++ side of
 * src/PyOrientationDistribution.hpp:458-600). */
class CustomOrientationDistribution : public OrientationDistribution {
public:
  CustomOrientationDistribution(const uint_fast32_t nmax,
                                double (*fn)(double, void *), void *arg)
      : OrientationDistribution(nmax) {
    compute(3, 0., fn, arg);
  }
};

/* Which orientation distribution a grain of a given size and shape follows
 * (src/AlignmentDistribution.hpp:35-52). */
class AlignmentDistribution {
public:
  virtual ~AlignmentDistribution() {}
  virtual const OrientationDistribution &
  get_distribution(const float_type equal_volume_radius,
                   const float_type axis_ratio) const = 0;
};

/* Grains above minimum_size align (oblate / prolate distribution by type:
 * 0 Davis-Greenstein, 1 Mishchenko, 2 disabled, 3 the given ones), smaller
 * grains orient randomly (src/SizeBasedAlignmentDistribution.hpp:68-146). */
class SizeBasedAlignmentDistribution : public AlignmentDistribution {
  float_type _minimum_size;
  OrientationDistribution *_random = nullptr, *_oblate = nullptr,
                          *_prolate = nullptr;

public:
  SizeBasedAlignmentDistribution(
      const float_type minimum_size,
      const int_fast32_t aligned_orientation_distribution_type,
      const uint_fast32_t nmax,
      const OrientationDistribution *oblate_aligned_orientation_distribution = nullptr,
      const OrientationDistribution *prolate_aligned_orientation_distribution = nullptr)
      : _minimum_size(minimum_size) {
    _random = new OrientationDistribution(2 * nmax);
    _random->initialise();
    switch (aligned_orientation_distribution_type) {
    case 0:
      _oblate = new DavisGreensteinOrientationDistribution(2 * nmax, 2.);
      _prolate = new DavisGreensteinOrientationDistribution(2 * nmax, 0.5);
      break;
    case 1:
      _oblate = new MishchenkoOrientationDistribution(2 * nmax, 0.6);
      _prolate = new MishchenkoOrientationDistribution(2 * nmax, 0.2);
      break;
    case 2:
      _oblate = new DisabledAlignmentOrientationDistribution();
      _prolate = new DisabledAlignmentOrientationDistribution();
      break;
    case 3:
      if (!oblate_aligned_orientation_distribution ||
          !prolate_aligned_orientation_distribution) {
        delete _random;
        throw std::runtime_error("tmx::SizeBasedAlignmentDistribution: type 3 "
                                 "needs oblate and prolate distributions");
      }
      // copies of the coefficients; averaging always on, as the reference's
      // OrientationDistribution copy constructor gives
      _oblate = new OrientationDistribution(*oblate_aligned_orientation_distribution);
      _prolate = new OrientationDistribution(*prolate_aligned_orientation_distribution);
      break;
    default:
      delete _random;
      throw std::runtime_error("tmx::SizeBasedAlignmentDistribution: unknown "
                               "orientation distribution");
    }
  }
  SizeBasedAlignmentDistribution(const SizeBasedAlignmentDistribution &) = delete;
  SizeBasedAlignmentDistribution &operator=(const SizeBasedAlignmentDistribution &) = delete;
  ~SizeBasedAlignmentDistribution() override {
    delete _random;
    delete _oblate;
    delete _prolate;
  }
  const OrientationDistribution &
  get_distribution(const float_type equal_volume_radius,
                   const float_type axis_ratio) const override {
    if (equal_volume_radius > _minimum_size) {
      return (axis_ratio > 1.) ? *_oblate : *_prolate;
    }
    return *_random;
  }
};

// ------------------------------------------------------------------- dust --

/* Refractive index of a grain (src/DustProperties.hpp:52-69). */
class DustProperties {
public:
  virtual ~DustProperties() {}
  virtual std::complex<float_type>
  get_refractive_index(const float_type wavelength, const float_type grain_size,
                       const int_fast32_t grain_type) const = 0;
};

/* Refractive index from a callback fn(wavelength, size, type, arg) (the C++
 * side of the module's CustomDustProperties, src/PyDustProperties.hpp). */
class CustomDustProperties : public DustProperties {
  std::complex<double> (*_fn)(double, double, int32_t, void *);
  void *_arg;

public:
  CustomDustProperties(std::complex<double> (*fn)(double, double, int32_t, void *),
                       void *arg = nullptr)
      : _fn(fn), _arg(arg) {}
  std::complex<float_type>
  get_refractive_index(const float_type wavelength, const float_type grain_size,
                       const int_fast32_t grain_type) const override {
    return _fn(wavelength, grain_size, (int32_t)grain_type, _arg);
  }
};

// ---------------------------------------------------------------- results --

/* Placeholders for the reference's graph objects: generate_tasks leaves the
 * task and resource lists empty and the space manager null. */
class Task {
public:
  virtual ~Task() {}
};
class Resource {
public:
  virtual ~Resource() {}
};
class TMatrixAuxiliarySpaceManager {};

/* Index of a result in the results list: (composition, size, wavelength,
 * result) in row-major order (src/ResultKey.hpp:38-156). Results of one
 * cell: extinction (if requested), absorption (if requested), scattering
 * matrices (if requested), in that order (TaskManager.hpp:460-472,
 * 1010-1060). */
class ResultKey {
  std::vector<int_fast32_t> _compositions;
  std::vector<float_type> _sizes, _wavelengths;
  uint_fast32_t _number_of_results;

public:
  ResultKey(const std::vector<int_fast32_t> &compositions,
            const std::vector<float_type> &sizes,
            const std::vector<float_type> &wavelengths,
            const uint_fast32_t number_of_results = 1)
      : _compositions(compositions), _sizes(sizes), _wavelengths(wavelengths),
        _number_of_results(number_of_results) {}
  size_t composition_size() const { return _compositions.size(); }
  size_t size_size() const { return _sizes.size(); }
  size_t wavelength_size() const { return _wavelengths.size(); }
  uint_fast32_t results_size() const { return _number_of_results; }
  int_fast32_t get_composition(const size_t index) const { return _compositions.at(index); }
  float_type get_size(const size_t index) const { return _sizes.at(index); }
  float_type get_wavelength(const size_t index) const { return _wavelengths.at(index); }
  size_t get_result_index(const size_t composition_index, const size_t size_index,
                          const size_t wavelength_index,
                          const uint_fast32_t result_index = 0) const {
    return composition_index * _sizes.size() * _wavelengths.size() * _number_of_results +
           size_index * _wavelengths.size() * _number_of_results +
           wavelength_index * _number_of_results + result_index;
  }
};

class Result {
public:
  virtual ~Result() {}
};

class AbsorptionCoefficientResult : public Result {
public:
  std::vector<float_type> Qabs, Qabspol; // per zenith angle
  float_type get_Qabs(const uint_fast32_t index) const { return Qabs.at(index); }
  float_type get_Qabspol(const uint_fast32_t index) const { return Qabspol.at(index); }
};

class ExtinctionCoefficientResult : public Result {
public:
  std::vector<float_type> Qext, Qextpol, Qextcpol; // per zenith angle
  float_type get_Qext(const uint_fast32_t index) const { return Qext.at(index); }
  float_type get_Qextpol(const uint_fast32_t index) const { return Qextpol.at(index); }
  float_type get_Qextcpol(const uint_fast32_t index) const { return Qextcpol.at(index); }
};

/* A 4 x 4 real matrix with the reference Matrix<float_type>'s accessor. */
struct Matrix4 {
  float_type m[16];
  float_type operator()(const uint_fast32_t row, const uint_fast32_t col) const {
    return m[4 * row + col];
  }
};

/* Scattering matrices on the reference's grid: index 2 ntheta * itheta +
 * iphi, theta_in = pi/2, ntheta Gauss-Legendre zenith and 2 ntheta
 * Gauss-Legendre azimuth angles (ScatteringMatrixTask.hpp:107-277). */
class ScatteringMatrixResult : public Result {
public:
  std::vector<Matrix4> Z;
  const Matrix4 &get_scattering_matrix(const uint_fast32_t index) const {
    return Z.at(index);
  }
};

// -------------------------------------------------------------- scheduler --

/* Handle with the shape of the reference's QuickSched wrapper
 * (src/QuickSchedWrapper.hpp:302-375): it owns a device context, and
 * execute_tasks() runs the batch the last generate_tasks() described. The
 * thread count is accepted for the interface and not used (one host thread
 * drives the device); graph logs are not written. */
class QuickSched {
public:
  /* what generate_tasks hands over */
  struct Batch {
    bool pending = false;
    std::vector<int32_t> types;
    std::vector<double> sizes, lambdas, thetas, shapes, weights, mr, mi, coeffs;
    std::vector<int32_t> orient_set;
    int32_t nsets = 0, ncoef = 0, flags = 0, ngauss = 20;
    tmx_schedule schedule = {10, 100, 2, 0, 1.e-4};
    std::vector<Result *> results; // not owned
    bool do_ext = false, do_abs = false, do_sca = false;
  };

  QuickSched(const int_fast32_t number_of_threads = 1, const bool graph_log = false,
             const std::string graph_log_name = "", const bool verbose = false,
             const int device = 0)
      : _threads(number_of_threads), _verbose(verbose) {
    (void)graph_log;
    (void)graph_log_name;
    if (tmx_create(&_ctx, device) != TMX_OK) {
      throw std::runtime_error("tmx::QuickSched: no usable CUDA device");
    }
  }
  QuickSched(const QuickSched &) = delete;
  QuickSched &operator=(const QuickSched &) = delete;
  ~QuickSched() { tmx_destroy(_ctx); }

  Batch &batch() { return _batch; }
  tmx_ctx *context() { return _ctx; }
  /* per-grain status bits of the last execute_tasks():
   * [composition][size][wavelength][shape] (tmx_grain_status) */
  const std::vector<int32_t> &grain_status() const { return _status; }

  void execute_tasks(const int_fast32_t number_of_threads = -1) {
    (void)number_of_threads;
    Batch &B = _batch;
    if (!B.pending) {
      return;
    }
    B.pending = false;
    const size_t nt = B.types.size(), ns = B.sizes.size(), nl = B.lambdas.size();
    const size_t nth = B.thetas.size(), nsh = B.shapes.size();
    const size_t ncell = nt * ns * nl;
    const int nq = (B.do_abs ? 2 : 0) + (B.do_ext ? 3 : 0);
    std::vector<double> q(std::max<size_t>(1, ncell * nth * std::max(nq, 1)));
    std::vector<double> z(B.do_sca ? ncell * nth * 2 * nth * 16 : 1);
    _status.assign(ncell * nsh, 0);
    const int rc = tmx_get_table(
        _ctx, (int32_t)nt, (int32_t)ns, B.sizes.data(), (int32_t)nl,
        B.lambdas.data(), (int32_t)nth, B.thetas.data(), (int32_t)nsh,
        B.shapes.data(), B.weights.data(), B.mr.data(), B.mi.data(),
        B.orient_set.data(), B.nsets, B.coeffs.data(), B.ncoef, B.flags,
        B.ngauss, &B.schedule, nq ? q.data() : nullptr,
        B.do_sca ? z.data() : nullptr, _status.data());
    if (rc != TMX_OK) {
      throw std::runtime_error(std::string("tmx::QuickSched::execute_tasks: ") +
                               tmx_last_error(_ctx));
    }
    // results per cell in the reference's order: extinction, absorption,
    // scattering
    const size_t per = (B.do_ext ? 1 : 0) + (B.do_abs ? 1 : 0) + (B.do_sca ? 1 : 0);
    for (size_t c = 0; c < ncell; ++c) {
      size_t r = c * per;
      const double *qc = q.data() + c * nth * std::max(nq, 1);
      const int ext0 = B.do_abs ? 2 : 0;
      if (B.do_ext) {
        auto *E = static_cast<ExtinctionCoefficientResult *>(B.results[r++]);
        E->Qext.resize(nth);
        E->Qextpol.resize(nth);
        E->Qextcpol.resize(nth);
        for (size_t t = 0; t < nth; ++t) {
          E->Qext[t] = qc[t * nq + ext0];
          E->Qextpol[t] = qc[t * nq + ext0 + 1];
          E->Qextcpol[t] = qc[t * nq + ext0 + 2];
        }
      }
      if (B.do_abs) {
        auto *A = static_cast<AbsorptionCoefficientResult *>(B.results[r++]);
        A->Qabs.resize(nth);
        A->Qabspol.resize(nth);
        for (size_t t = 0; t < nth; ++t) {
          A->Qabs[t] = qc[t * nq];
          A->Qabspol[t] = qc[t * nq + 1];
        }
      }
      if (B.do_sca) {
        auto *S = static_cast<ScatteringMatrixResult *>(B.results[r++]);
        const size_t nz = nth * 2 * nth;
        S->Z.resize(nz);
        for (size_t k = 0; k < nz; ++k) {
          std::copy(z.data() + (c * nz + k) * 16, z.data() + (c * nz + k + 1) * 16,
                    S->Z[k].m);
        }
      }
    }
  }

private:
  tmx_ctx *_ctx = nullptr;
  int_fast32_t _threads;
  bool _verbose;
  Batch _batch;
  std::vector<int32_t> _status;
};

// ------------------------------------------------------------ TaskManager --

/* The reference's TaskManager (src/TaskManager.hpp:371-455): the grid of
 * compositions x sizes x wavelengths (x the shape distribution's nodes) and
 * the convergence schedule. */
class TaskManager {
  uint_fast32_t _minimum_order, _maximum_order, _gauss_legendre_factor;
  float_type _tolerance;
  size_t _maximum_memory_usage;
  const ShapeDistribution &_shape_distribution;
  const AlignmentDistribution &_alignment_distribution;
  const DustProperties &_dust_properties;
  std::vector<int_fast32_t> _compositions;
  std::vector<float_type> _sizes, _wavelengths;

public:
  TaskManager(const uint_fast32_t minimum_order, const uint_fast32_t maximum_order,
              const uint_fast32_t gauss_legendre_factor, const float_type tolerance,
              const size_t maximum_memory_usage,
              const ShapeDistribution &shape_distribution,
              const AlignmentDistribution &alignment_distribution,
              const DustProperties &dust_properties)
      : _minimum_order(minimum_order), _maximum_order(maximum_order),
        _gauss_legendre_factor(gauss_legendre_factor), _tolerance(tolerance),
        _maximum_memory_usage(maximum_memory_usage),
        _shape_distribution(shape_distribution),
        _alignment_distribution(alignment_distribution),
        _dust_properties(dust_properties) {}

  void add_composition(const int_fast32_t composition) {
    _compositions.push_back(composition);
  }
  void add_size(const float_type size) { _sizes.push_back(size); }
  void add_wavelength(const float_type wavelength) {
    _wavelengths.push_back(wavelength);
  }

  /* Describes the whole grid as one device batch on `quicksched` (sizes and
   * wavelengths sorted, as the reference sorts them). tasks, resources and
   * space_manager are left empty / null; result_key and results are new
   * objects that the caller deletes after reading them, as in the
   * reference. The memory limit and the memory log are accepted and not
   * used: the device path bounds its own work in chunks. */
  void generate_tasks(const std::vector<float_type> &theta, const uint_fast32_t ngauss,
                      QuickSched &quicksched, std::vector<Task *> &tasks,
                      std::vector<Resource *> &resources, ResultKey *&result_key,
                      std::vector<Result *> &results,
                      TMatrixAuxiliarySpaceManager *&space_manager,
                      const bool do_extinction, const bool do_absorption,
                      const bool do_scattering, const bool account_for_scattering,
                      const bool verbose = false, const bool write_memory_log = false,
                      const std::string memory_log_file_name = "") {
    (void)tasks;
    (void)resources;
    (void)verbose;
    (void)write_memory_log;
    (void)memory_log_file_name;
    space_manager = nullptr;
    std::sort(_sizes.begin(), _sizes.end());
    std::sort(_wavelengths.begin(), _wavelengths.end());
    const size_t nt = _compositions.size(), ns = _sizes.size(), nl = _wavelengths.size();
    const uint_fast32_t nres = (do_extinction ? 1 : 0) + (do_absorption ? 1 : 0) +
                               (do_scattering ? 1 : 0);
    result_key = new ResultKey(_compositions, _sizes, _wavelengths, nres);
    QuickSched::Batch &B = quicksched.batch();
    B = QuickSched::Batch();
    B.types.assign(_compositions.begin(), _compositions.end());
    B.sizes = _sizes;
    B.lambdas = _wavelengths;
    B.thetas = theta;
    const uint_fast32_t nsh = _shape_distribution.get_number_of_points();
    for (uint_fast32_t i = 0; i < nsh; ++i) {
      B.shapes.push_back(_shape_distribution.get_shape(i));
      B.weights.push_back(_shape_distribution.get_weight(i));
    }
    // refractive index of every (composition, size, wavelength) cell
    B.mr.resize(nt * ns * nl);
    B.mi.resize(nt * ns * nl);
    for (size_t it = 0; it < nt; ++it) {
      for (size_t is = 0; is < ns; ++is) {
        for (size_t il = 0; il < nl; ++il) {
          const std::complex<float_type> m = _dust_properties.get_refractive_index(
              _wavelengths[il], _sizes[is], _compositions[it]);
          B.mr[(it * ns + is) * nl + il] = m.real();
          B.mi[(it * ns + is) * nl + il] = m.imag();
        }
      }
    }
    // orientation coefficient set of every (size, shape)
    std::vector<const OrientationDistribution *> sets;
    B.orient_set.assign(ns * nsh, -1);
    size_t ncoef = 2 * (size_t)_maximum_order + 1;
    for (size_t is = 0; is < ns; ++is) {
      for (uint_fast32_t ish = 0; ish < nsh; ++ish) {
        const OrientationDistribution &od =
            _alignment_distribution.get_distribution(_sizes[is], B.shapes[ish]);
        if (!od.compute_alignment()) {
          continue;
        }
        size_t k = 0;
        while (k < sets.size() && sets[k] != &od) {
          ++k;
        }
        if (k == sets.size()) {
          sets.push_back(&od);
          ncoef = std::max(ncoef, od.coefficients().size());
        }
        B.orient_set[is * nsh + ish] = (int32_t)k;
      }
    }
    B.nsets = (int32_t)sets.size();
    B.ncoef = (int32_t)ncoef;
    B.coeffs.assign(std::max<size_t>(1, sets.size()) * ncoef, 0.);
    for (size_t k = 0; k < sets.size(); ++k) {
      const std::vector<float_type> &c = sets[k]->coefficients();
      std::copy(c.begin(), c.end(), B.coeffs.begin() + k * ncoef);
    }
    B.flags = (do_absorption ? TMX_TABLE_ABSORPTION : 0) |
              (do_extinction ? TMX_TABLE_EXTINCTION : 0) |
              (do_scattering ? TMX_TABLE_SCATTERING : 0) |
              (account_for_scattering ? TMX_TABLE_ACCOUNT_FOR_SCATTERING : 0);
    B.ngauss = (int32_t)ngauss;
    B.schedule.min_order = (int32_t)_minimum_order;
    B.schedule.max_order = (int32_t)_maximum_order;
    B.schedule.gauss_legendre_factor = (int32_t)_gauss_legendre_factor;
    B.schedule.bessel_start = 0;
    B.schedule.tolerance = _tolerance;
    B.do_ext = do_extinction;
    B.do_abs = do_absorption;
    B.do_sca = do_scattering;
    results.assign(nt * ns * nl * nres, nullptr);
    for (size_t c = 0; c < nt * ns * nl; ++c) {
      size_t r = c * nres;
      if (do_extinction) {
        results[r++] = new ExtinctionCoefficientResult();
      }
      if (do_absorption) {
        results[r++] = new AbsorptionCoefficientResult();
      }
      if (do_scattering) {
        results[r++] = new ScatteringMatrixResult();
      }
    }
    B.results = results;
    B.pending = true;
  }
};

} // namespace tmx

#endif // TMX_TASKMANAGER_HPP
