// C-ABI harness around the unmodified CosTuuM reference (test infrastructure).
//
// This file is compiled by oracle/build_ref.sh against the reference's own
// headers (nothing of the reference is copied here). It exposes:
//   * stage-level entry points (Gauss-Legendre rule, spherical Bessel arrays,
//     Wigner d arrays, Clebsch-Gordan rows, plu_inverse, orientation
//     distribution coefficients) used to pin the C restatement in
//     oracle/tmx_oracle.c bit for bit where the arithmetic order allows;
//   * a batch entry point that wires the reference's task objects for many
//     independent grains exactly like TaskManager::generate_tasks wires one
//     grain's convergence chain (src/TaskManager.hpp:1146-1197, MAll tasks
//     :1313-1327) and runs them under the reference's QuickSched. This is the
//     "reference QuickSched CPU path" that the benchmark's reference arm times.
//
// Only tests/, the golden-fixture script and bench.py's CPU-baseline leg load
// the resulting library.

#include "Configuration.hpp"

#include "AlignmentAverageTask.hpp"
#include "ConvergedSizeResources.hpp"
#include "DavisGreensteinOrientationDistribution.hpp"
#include "DraineHensleyShapeDistribution.hpp"
#include "GaussBasedResources.hpp"
#include "InteractionResource.hpp"
#include "Matrix.hpp"
#include "MishchenkoOrientationDistribution.hpp"
#include "NBasedResources.hpp"
#include "OrientationDistribution.hpp"
#include "ParticleGeometryResource.hpp"
#include "QuickSchedWrapper.hpp"
#include "SpecialFunctions.hpp"
#include "TMatrixResource.hpp"
#include "WignerDResources.hpp"

#include <complex>
#include <cstring>
#include <vector>

extern "C" {

// ---------------------------------------------------------------- stages ---

void ref_gauss_legendre(int order, double *x, double *w) {
  std::vector<double> px(order), pw(order);
  SpecialFunctions::get_gauss_legendre_points_and_weights(order, px, pw);
  for (int i = 0; i < order; ++i) {
    x[i] = px[i];
    w[i] = pw[i];
  }
}

void ref_bessel_j_real(int nmax, double z, double *j, double *dj) {
  SpecialFunctions::spherical_j_jdj_array<double>(nmax, z, j, dj);
}

void ref_bessel_y_real(int nmax, double z, double *y, double *dy) {
  SpecialFunctions::spherical_y_ydy_array<double>(nmax, z, y, dy);
}

// complex arrays are interleaved (re, im)
void ref_bessel_j_complex(int nmax, double zr, double zi, double *j,
                          double *dj) {
  std::vector<std::complex<double>> cj(nmax), cdj(nmax);
  SpecialFunctions::spherical_j_jdj_array<std::complex<double>>(
      nmax, std::complex<double>(zr, zi), &cj[0], &cdj[0]);
  for (int i = 0; i < nmax; ++i) {
    j[2 * i] = cj[i].real();
    j[2 * i + 1] = cj[i].imag();
    dj[2 * i] = cdj[i].real();
    dj[2 * i + 1] = cdj[i].imag();
  }
}

void ref_wigner_d(double cosx, int nmax, int m, double *d, double *dd) {
  SpecialFunctions::wigner_dn_0m<double>(cosx, nmax, m, d, dd);
}

void ref_wigner_d_sinx(double cosx, double sinx, double sinx_inv, int nmax,
                       int m, double *d, double *dd) {
  SpecialFunctions::wigner_dn_0m_sinx<double>(cosx, sinx, sinx_inv, nmax, m, d,
                                              dd);
}

double ref_rv_over_rs(double axis_ratio) {
  return SpecialFunctions::get_equal_volume_to_equal_surface_area_sphere_ratio(
      axis_ratio);
}

// returns the number of coefficients written (2 min(n1,n2) + 1); C must hold
// (N + 1) (2 n1 + 1) doubles of scratch
int ref_clebsch_gordan_row(int n1, int n2, int N, double *C) {
  std::vector<double> c((N + 1) * (2 * n1 + 1), 0.);
  const int n =
      SpecialFunctions::get_clebsch_gordan_coefficients<double>(n1, n2, N, c);
  for (int i = 0; i < n; ++i) {
    C[i] = c[i];
  }
  return n;
}

double ref_clebsch_gordan(int n1, int m1, int n2, int m2, int N, int M) {
  return SpecialFunctions::get_clebsch_gordan_coefficient<double>(n1, m1, n2,
                                                                  m2, N, M);
}

// in-place inverse of an n x n complex matrix (row major, interleaved)
void ref_plu_inverse(int n, double *a) {
  Matrix<std::complex<double>> A(n, n);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      A(i, j) = std::complex<double>(a[2 * (i * n + j)], a[2 * (i * n + j) + 1]);
    }
  }
  A.plu_inverse(n);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      a[2 * (i * n + j)] = A(i, j).real();
      a[2 * (i * n + j) + 1] = A(i, j).imag();
    }
  }
}

// kind: 0 random (numerical quadrature), 1 Mishchenko(param = cos2beta),
//       2 Davis-Greenstein(param = axis ratio); writes order + 1 coefficients
void ref_orientation_coefficients(int kind, double param, int order,
                                  double *out) {
  OrientationDistribution *od = nullptr;
  if (kind == 0) {
    od = new OrientationDistribution(order);
    od->initialise();
  } else if (kind == 1) {
    od = new MishchenkoOrientationDistribution(order, param);
  } else {
    od = new DavisGreensteinOrientationDistribution(order, param);
  }
  for (int i = 0; i <= order; ++i) {
    out[i] = od->get_coefficient(i);
  }
  delete od;
}

// an orientation distribution with a user-defined p(beta), initialised with
// the tolerances the Python module's custom distribution uses
// (PyOrientationDistribution.hpp: initialise(1e-4, 1e-4))
class RefCustomOrientation : public OrientationDistribution {
public:
  RefCustomOrientation(int order) : OrientationDistribution(order) {
    initialise(1.e-4, 1.e-4);
  }
  virtual float_type operator()(const float_type beta, const float_type cosbeta,
                                const float_type sinbeta) const {
    return 0.5 + 0.3 * cosbeta * cosbeta;
  }
};

// p(beta) = 0.5 + 0.3 cos^2(beta)
void ref_custom_orientation_coefficients(int order, double *out) {
  RefCustomOrientation od(order);
  for (int i = 0; i <= order; ++i) {
    out[i] = od.get_coefficient(i);
  }
}

// nodes, weights and limits of DraineHensleyShapeDistribution(npoints,
// cutoff, fraction)
void ref_draine_hensley(int npoints, double cutoff, double fraction,
                        double *shapes, double *weights, double *limits) {
  DraineHensleyShapeDistribution sd(npoints, cutoff, fraction);
  for (int i = 0; i < npoints; ++i) {
    shapes[i] = sd.get_shape(i);
    weights[i] = sd.get_weight(i);
  }
  limits[0] = sd.get_minimum_axis_ratio();
  limits[1] = sd.get_maximum_axis_ratio();
}

// ----------------------------------------------------------------- batch ---

struct RefBatch {
  int n;
  int min_order, max_order, glfac;
  QuickSched *qs;
  NBasedResources *nfactors;
  TMatrixAuxiliarySpaceManager *aux;
  std::vector<GaussBasedResources *> quad;
  std::vector<WignerDResources *> wigner;
  std::vector<ParticleGeometryResource *> geometry;
  std::vector<InteractionVariables *> ivars;
  std::vector<InteractionResource *> interactions;
  std::vector<ConvergedSizeResources *> converged;
  std::vector<TMatrixResource *> tmatrix;
  std::vector<Task *> tasks;
  std::vector<double> chain_qsca, chain_qext;
};

// r_ev, wavelength in metres; one independent grain per entry
void *ref_batch_create(int n, const double *r_ev, const double *wavelength,
                       const double *mr, const double *mi,
                       const double *axis_ratio, int min_order, int max_order,
                       int glfac, double tolerance, int nthreads) {
  RefBatch *b = new RefBatch();
  b->n = n;
  b->min_order = min_order;
  b->max_order = max_order;
  b->glfac = glfac;
  b->qs = new QuickSched(nthreads, false, "", false);
  QuickSched &qs = *b->qs;
  const int norders = max_order - min_order;

  b->nfactors = new NBasedResources(max_order);
  qs.register_resource(*b->nfactors);
  qs.register_task(*b->nfactors);
  b->nfactors->link_resources(qs);
  b->aux = new TMatrixAuxiliarySpaceManager(nthreads, max_order);

  for (int i = 0; i < norders; ++i) {
    const int order = min_order + i;
    GaussBasedResources *q = new GaussBasedResources(glfac * order);
    qs.register_resource(*q);
    qs.register_task(*q);
    q->link_resources(qs);
    b->quad.push_back(q);
    WignerDResources *w =
        new WignerDResources(order, glfac * order, *q, order < 100);
    qs.register_resource(*w);
    qs.register_task(*w);
    w->link_resources(qs);
    qs.link_tasks(*q, *w);
    b->wigner.push_back(w);
  }

  for (int g = 0; g < n; ++g) {
    InteractionVariables *iv = new InteractionVariables(
        r_ev[g], wavelength[g], std::complex<double>(mr[g], mi[g]));
    qs.register_resource(*iv);
    b->ivars.push_back(iv);
    InteractionResource *ir =
        new InteractionResource(max_order, glfac * max_order);
    qs.register_resource(*ir);
    b->interactions.push_back(ir);
    ConvergedSizeResources *cs = new ConvergedSizeResources();
    qs.register_resource(*cs);
    b->converged.push_back(cs);
    TMatrixResource *T = new TMatrixResource(max_order);
    qs.register_resource(*T);
    for (int m = 0; m < max_order + 1; ++m) {
      qs.register_resource(T->get_m_resource(m), T);
    }
    b->tmatrix.push_back(T);

    TMatrixM0Task *previous = nullptr;
    for (int i = 0; i < norders; ++i) {
      const int order = min_order + i;
      const int ng = glfac * order;
      ParticleGeometryResource *geo =
          new ParticleGeometryResource(axis_ratio[g], ng, *b->quad[i]);
      qs.register_resource(*geo);
      qs.register_task(*geo);
      geo->link_resources(qs);
      qs.link_tasks(*b->quad[i], *geo);
      b->geometry.push_back(geo);

      InteractionTask *it = new InteractionTask(order, ng, *geo, *cs, *iv, *ir);
      qs.register_task(*it);
      it->link_resources(qs);
      qs.link_tasks(*geo, *it);
      b->tasks.push_back(it);

      TMatrixM0Task *m0 = new TMatrixM0Task(
          tolerance, order, ng, *b->nfactors, *b->quad[i], *geo, *iv, *ir,
          *b->wigner[i], *b->aux, *T, *cs, T->get_m_resource(0));
      qs.register_task(*m0);
      m0->link_resources(qs);
      qs.link_tasks(*b->nfactors, *m0);
      qs.link_tasks(*b->wigner[i], *m0);
      qs.link_tasks(*it, *m0);
      if (previous != nullptr) {
        qs.link_tasks(*previous, *it);
        qs.link_tasks(*previous, *m0);
      }
      b->tasks.push_back(m0);
      previous = m0;
    }
    for (int m = 1; m <= max_order; ++m) {
      TMatrixMAllTask *ma = new TMatrixMAllTask(
          m, *b->nfactors, *cs, *iv, *ir, *b->aux, *T, T->get_m_resource(m));
      qs.register_task(*ma);
      ma->link_resources(qs);
      qs.link_tasks(*previous, *ma);
      b->tasks.push_back(ma);
    }
  }
  return b;
}

void ref_batch_run(void *h) {
  RefBatch *b = static_cast<RefBatch *>(h);
  b->qs->execute_tasks();
  b->chain_qsca.resize(b->n);
  b->chain_qext.resize(b->n);
  for (int g = 0; g < b->n; ++g) {
    // m = 0 sums of the converged order, as the convergence test saw them
    b->chain_qsca[g] = b->tmatrix[g]->get_scattering_coefficient();
    b->chain_qext[g] = b->tmatrix[g]->get_extinction_coefficient();
    // full sums over every m block (TMatrixQTask)
    TMatrixQTask q(*b->tmatrix[g]);
    q.execute(0);
  }
}

int ref_batch_nmax(void *h, int g) {
  return static_cast<RefBatch *>(h)->tmatrix[g]->get_nmax();
}

int ref_batch_ngauss(void *h, int g) {
  return static_cast<RefBatch *>(h)->tmatrix[g]->get_ngauss();
}

int ref_batch_converged(void *h, int g) {
  return static_cast<RefBatch *>(h)->converged[g]->is_converged() ? 1 : 0;
}

// out: [chain Qsca, chain Qext, full Qsca, full Qext, dQs, dQe]
void ref_batch_q(void *h, int g, double *out) {
  RefBatch *b = static_cast<RefBatch *>(h);
  out[0] = b->chain_qsca[g];
  out[1] = b->chain_qext[g];
  out[2] = b->tmatrix[g]->get_scattering_coefficient();
  out[3] = b->tmatrix[g]->get_extinction_coefficient();
  out[4] = b->converged[g]->get_dQs();
  out[5] = b->converged[g]->get_dQe();
}

// T block m of grain g as a (2 nb) x (2 nb) complex matrix, nb = nmax for
// m = 0 and nmax + 1 - m otherwise, in the reference's own index map
// (TMatrixResource::operator(), src/TMatrixResource.hpp:195-213)
void ref_batch_tblock(void *h, int g, int m, double *out) {
  RefBatch *b = static_cast<RefBatch *>(h);
  const TMatrixResource &T = *b->tmatrix[g];
  const int nmax = T.get_nmax();
  const int nmin = (m > 0) ? m : 1;
  const int nb = nmax + 1 - nmin;
  for (int i1 = 0; i1 < 2; ++i1) {
    for (int n1 = nmin; n1 <= nmax; ++n1) {
      for (int i2 = 0; i2 < 2; ++i2) {
        for (int n2 = nmin; n2 <= nmax; ++n2) {
          const std::complex<double> v = T(i1, n1, m, i2, n2, m);
          const int r = i1 * nb + (n1 - nmin);
          const int c = i2 * nb + (n2 - nmin);
          out[2 * (r * 2 * nb + c)] = v.real();
          out[2 * (r * 2 * nb + c) + 1] = v.imag();
        }
      }
    }
  }
}

void ref_batch_destroy(void *h) {
  RefBatch *b = static_cast<RefBatch *>(h);
  for (Task *t : b->tasks) {
    delete t;
  }
  for (auto *p : b->geometry) {
    delete p;
  }
  for (auto *p : b->ivars) {
    delete p;
  }
  for (auto *p : b->interactions) {
    delete p;
  }
  for (auto *p : b->converged) {
    delete p;
  }
  for (auto *p : b->tmatrix) {
    delete p;
  }
  for (auto *p : b->wigner) {
    delete p;
  }
  for (auto *p : b->quad) {
    delete p;
  }
  delete b->nfactors;
  delete b->aux;
  delete b->qs;
  delete b;
}

} // extern "C"
