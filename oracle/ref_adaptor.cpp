/*
 * ref_adaptor.cpp -- C entry points over the drop-in adaptor B200FrameWarper
 * (frame-aligner_b200/adaptor/B200FrameWarper.h) driven by the reference's own classes (TEST
 * INFRASTRUCTURE ONLY). oracle/Makefile compiles the reference's FrameWarper.cpp (the non-virtual
 * AbstractFrameWarper::setReference that calls the adaptor's setupReferenceInformation hook),
 * Sobel3d.cpp and OptimisationModel.cpp unchanged against the container stand-ins in ref_shim/,
 * together with this file and the adaptor header, into oracle/_ref/libfa_adaptor.so, linked to
 * frame-aligner_b200/libfa_b200.so. Tests compare what the reference's OptimisationModel reads
 * through the adaptor (f, J^T e, H) and the solve it drives with the reference's CpuFrameWarper.
 */
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "B200FrameWarper.h"
#include "OptimisationModel.h"

extern "C" {
#include "fa_oracle.h"
}

// Axis indices of the reference's dims convention (FrameAligner/Cv3dUtils.cpp:6-8), which the
// reference headers declare and Cv3dUtils.cpp (not part of this build) defines.
const int X = 2;
const int Y = 1;
const int Z = 0;

namespace {

struct Adaptor {
  std::shared_ptr<B200FrameWarper> w;
  cv::Mat frame;  // the registered frame (identified by its data pointer)
  int nz, ny, nx, nD;
};

cv::Mat make_mat(const float* data, int nz, int ny, int nx) {
  cv::Mat m(std::vector<int>{nz, ny, nx}, CV_32F);
  std::memcpy(m.data, data, sizeof(float) * (size_t)nz * ny * nx);
  return m;
}

column_vector to_col(const double* D, int nD, int nd) {
  std::vector<cv::Point3d> v((size_t)nD);
  for (int i = 0; i < nD; i++) v[(size_t)i] = cv::Point3d(D[3 * i], D[3 * i + 1], D[3 * i + 2]);
  column_vector c;
  D2col(v, c, nd);
  return c;
}

struct ModelCtx {
  OptimisationModel* model;
  int P;
};

double f_cb(void* ctx, const double* x) {
  ModelCtx* c = static_cast<ModelCtx*>(ctx);
  column_vector v;
  v.set_size(c->P);
  for (int i = 0; i < c->P; i++) v(i) = x[i];
  return (*c->model)(v);
}

void g_cb(void* ctx, const double* x, double* g) {
  ModelCtx* c = static_cast<ModelCtx*>(ctx);
  column_vector v, der;
  v.set_size(c->P);
  for (int i = 0; i < c->P; i++) v(i) = x[i];
  dlib::matrix<double> hess;
  c->model->get_derivative_and_hessian(v, der, hess);
  for (int i = 0; i < c->P; i++) g[i] = der(i);
}

}  // namespace

extern "C" {

// B200FrameWarper::getGpuSupportInformation: 1 when supported, message copied into msg.
int fa_adaptor_gpu_support(char* msg, int len) {
  GpuSupportInformation s = B200FrameWarper::getGpuSupportInformation();
  std::snprintf(msg, (size_t)len, "%s", s.message.c_str());
  return s.supported ? 1 : 0;
}

// new B200FrameWarper + the reference's AbstractFrameWarper::setReference (FrameWarper.cpp:186-205).
void* fa_adaptor_create(const float* ref, int nz, int ny, int nx, int nD, double line, double interline,
                        double interframe, int bidirectional, int precision, char* err) {
  try {
    ImageScanParameters sp(line, interline, interframe, nx, ny, nz, bidirectional != 0);
    sp.bidirectional = bidirectional != 0;  // the reference constructor does not store it
    Adaptor* a = new Adaptor;
    a->w = std::make_shared<B200FrameWarper>(0, precision ? FA_PREC_MIXED : FA_PREC_F32);
    a->nz = nz;
    a->ny = ny;
    a->nx = nx;
    a->nD = nD;
    a->w->setReference(make_mat(ref, nz, ny, nx), nD, sp);
    return a;
  } catch (std::exception& e) {
    if (err) std::snprintf(err, 256, "%s", e.what());
    return nullptr;
  }
}

void fa_adaptor_destroy(void* h) { delete static_cast<Adaptor*>(h); }

int fa_adaptor_n_dim(void* h) { return static_cast<Adaptor*>(h)->w->n_dim; }

// registerFrame (the previous frame is deregistered first, as addFrame does, FrameWarpAligner.cpp:223)
int fa_adaptor_set_frame(void* h, const float* frame, char* err) {
  Adaptor* a = static_cast<Adaptor*>(h);
  try {
    if (!a->frame.empty()) a->w->deregisterFrame(a->frame);
    a->frame = make_mat(frame, a->nz, a->ny, a->nx);
    a->w->registerFrame(a->frame);
    return 0;
  } catch (std::exception& e) {
    if (err) std::snprintf(err, 256, "%s", e.what());
    return 1;
  }
}

// OptimisationModel::operator() and get_derivative_and_hessian (OptimisationModel.cpp:45-62) over
// the adaptor at D (nD x 3): f, der (P doubles) and hess (P x P) as the model sees them.
int fa_adaptor_model(void* h, const double* D, double* f, double* der, double* hess, char* err) {
  Adaptor* a = static_cast<Adaptor*>(h);
  try {
    OptimisationModel model(a->w, a->frame);
    const int nd = a->w->n_dim, P = a->nD * nd;
    column_vector x = to_col(D, a->nD, nd), d;
    *f = model(x);
    dlib::matrix<double> H;
    model.get_derivative_and_hessian(x, d, H);
    for (int i = 0; i < P; i++) der[i] = d(i);
    for (int i = 0; i < P * P; i++) hess[i] = H.data()[i];
    return 0;
  } catch (std::exception& e) {
    if (err) std::snprintf(err, 256, "%s", e.what());
    return 1;
  }
}

// warpImageInterpolated through the adaptor.
int fa_adaptor_warp(void* h, const double* D, int invalid_value, float* out, char* err) {
  Adaptor* a = static_cast<Adaptor*>(h);
  try {
    std::vector<cv::Point3d> v((size_t)a->nD);
    for (int i = 0; i < a->nD; i++) v[(size_t)i] = cv::Point3d(D[3 * i], D[3 * i + 1], D[3 * i + 2]);
    cv::Mat wimg;
    a->w->warpImageInterpolated(a->frame, wimg, v, invalid_value);
    std::memcpy(out, wimg.data, sizeof(float) * (size_t)a->nz * a->ny * a->nx);
    return 0;
  } catch (std::exception& e) {
    if (err) std::snprintf(err, 256, "%s", e.what());
    return 1;
  }
}

// The solve of FrameWarpAligner::addFrame (FrameWarpAligner.cpp:147-219) with the reference's
// OptimisationModel over the adaptor: starting points {0, 0, rigid}, the first minimum, then the
// project's trust region (dlib is not in the reference tree) with the H the model reads.
int fa_adaptor_align(void* h, const double* rigid, int max_iter, double* D_out, int* iters, char* err) {
  Adaptor* a = static_cast<Adaptor*>(h);
  try {
    OptimisationModel model(a->w, a->frame);
    const int nd = a->w->n_dim, P = a->nD * nd;
    ModelCtx ctx{&model, P};
    std::vector<std::vector<double>> start(3, std::vector<double>((size_t)P, 0.0));
    for (int i = 0; i < a->nD; i++)
      for (int c = 0; c < nd; c++) start[2][(size_t)(i * nd + c)] = rigid[c];
    double fe[3];
    for (int s = 0; s < 3; s++) fe[s] = f_cb(&ctx, start[(size_t)s].data());
    int best = 0;
    for (int s = 1; s < 3; s++)
      if (fe[s] < fe[best]) best = s;
    std::vector<double> x = start[(size_t)best];
    // the H the model hands the solver (the adaptor's warper->H, OptimisationModel.cpp:61)
    column_vector xc, der;
    dlib::matrix<double> H;
    xc.set_size(P);
    for (int i = 0; i < P; i++) xc(i) = x[(size_t)i];
    model.get_derivative_and_hessian(xc, der, H);
    or_tr_stats st;
    or_trust_region(P, H.data(), x.data(), 40.0, 1e-8, max_iter, f_cb, g_cb, &ctx, &st);
    for (int i = 0; i < a->nD; i++) {
      D_out[3 * i] = x[(size_t)(i * nd)];
      D_out[3 * i + 1] = x[(size_t)(i * nd + 1)];
      D_out[3 * i + 2] = nd == 3 ? x[(size_t)(i * nd + 2)] : 0.0;
    }
    if (iters) *iters = st.iterations;
    return 0;
  } catch (std::exception& e) {
    if (err) std::snprintf(err, 256, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
