/*
 * ref_wrap.cpp -- C entry points over the reference's OWN warper sources (TEST INFRASTRUCTURE
 * ONLY). oracle/Makefile compiles FrameWarper.cpp, Sobel3d.cpp, VolumePhaseCorrelator.cpp and
 * OptimisationModel.cpp unchanged from the reference tree (FrameAligner/), against the
 * container stand-ins in oracle/ref_shim/, and links them with this file into
 * oracle/_ref/libfa_ref.so. Tests use it to pin the C restatement (fa_oracle.c) bit for bit, and
 * bench.py's reference arm times it as the reference CPU path.
 *
 * The trust-region driver is the oracle's (fa_oracle_tr.c): dlib is not part of the reference
 * tree. Everything else on the per-frame path -- CpuFrameWarper::getError / getJacobian,
 * OptimisationModel, VolumePhaseCorrelator -- is the reference's code.
 */
#include <pthread.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "FrameWarper.h"
#include "OptimisationModel.h"
#include "Sobel3d.h"
#include "VolumePhaseCorrelator.h"

extern "C" {
#include "fa_oracle.h"
}

// Axis indices of the reference's dims convention (FrameAligner/Cv3dUtils.cpp:6-8).
const int X = 2;
const int Y = 1;
const int Z = 0;

namespace {

// Exposes the protected precomputed state of the reference warper for comparison.
class RefWarper : public CpuFrameWarper {
 public:
  const cv::Mat& di() const { return Di; }
  const cv::Mat& df() const { return Df; }
  const std::vector<Range>& ranges() const { return D_range; }
  const dlib::matrix<double>& hess() const { return H; }
};

struct Handle {
  std::shared_ptr<RefWarper> w;
  cv::Mat frame;  // stable storage: the reference keys its error buffer on frame.data
  int nz, ny, nx, nD;
};

cv::Mat make_mat(const float* data, int nz, int ny, int nx) {
  cv::Mat m(std::vector<int>{nz, ny, nx}, CV_32F);
  std::memcpy(m.data, data, sizeof(float) * (size_t)nz * ny * nx);
  return m;
}

std::vector<cv::Point3d> to_points(const double* D, int nD) {
  std::vector<cv::Point3d> v((size_t)nD);
  for (int i = 0; i < nD; i++) v[(size_t)i] = cv::Point3d(D[3 * i], D[3 * i + 1], D[3 * i + 2]);
  return v;
}

Handle* create(const float* ref, int nz, int ny, int nx, int nD, double line, double interline, double interframe,
               int bidirectional, char* err) {
  try {
    ImageScanParameters sp(line, interline, interframe, nx, ny, nz, bidirectional != 0);
    sp.bidirectional = bidirectional != 0;  // the reference constructor does not store it
    Handle* h = new Handle;
    h->w = std::make_shared<RefWarper>();
    h->nz = nz;
    h->ny = ny;
    h->nx = nx;
    h->nD = nD;
    h->w->setReference(make_mat(ref, nz, ny, nx), nD, sp);
    return h;
  } catch (std::exception& e) {
    if (err) std::snprintf(err, 128, "%s", e.what());
    return nullptr;
  }
}

}  // namespace

extern "C" {

void* fr_warper_create(const float* ref, int nz, int ny, int nx, int nD, double line, double interline,
                       double interframe, int bidirectional, char* err) {
  return create(ref, nz, ny, nx, nD, line, interline, interframe, bidirectional, err);
}

void fr_warper_destroy(void* hp) { delete static_cast<Handle*>(hp); }

int fr_n_dim(void* hp) { return static_cast<Handle*>(hp)->w->n_dim; }

void fr_set_frame(void* hp, const float* frame) {
  Handle* h = static_cast<Handle*>(hp);
  h->frame = make_mat(frame, h->nz, h->ny, h->nx);
}

double fr_get_error(void* hp, const double* D) {
  Handle* h = static_cast<Handle*>(hp);
  return h->w->getError(h->frame, to_points(D, h->nD));
}

void fr_get_jacobian(void* hp, const double* D, double* jac) {
  Handle* h = static_cast<Handle*>(hp);
  column_vector j;
  h->w->getJacobian(h->frame, to_points(D, h->nD), j);
  for (long i = 0; i < j.size(); i++) jac[i] = j(i);
}

// H read the way OptimisationModel does (OptimisationModel.cpp:55-62).
void fr_hessian(void* hp, double* H) {
  Handle* h = static_cast<Handle*>(hp);
  OptimisationModel model(h->w, h->frame);
  int P = h->nD * h->w->n_dim;
  column_vector x, der;
  x.set_size(P);
  dlib::matrix<double> hess;
  // get_derivative_and_hessian needs an error buffer for the frame: evaluate at x = 0 first.
  model(x);
  model.get_derivative_and_hessian(x, der, hess);
  for (int i = 0; i < P * P; i++) H[i] = hess.data()[i];
}

double fr_model_f(void* hp, const double* x) {
  Handle* h = static_cast<Handle*>(hp);
  OptimisationModel model(h->w, h->frame);
  int P = h->nD * h->w->n_dim;
  column_vector c;
  c.set_size(P);
  for (int i = 0; i < P; i++) c(i) = x[i];
  return model(c);
}

void fr_precomp(void* hp, uint16_t* Di, float* Df, int* ranges) {
  Handle* h = static_cast<Handle*>(hp);
  size_t N = (size_t)h->nz * h->ny * h->nx;
  std::memcpy(Di, h->w->di().data, N * sizeof(uint16_t));
  std::memcpy(Df, h->w->df().data, N * sizeof(float));
  for (int k = 0; k < h->nD; k++) {
    ranges[2 * k] = h->w->ranges()[(size_t)k].begin;
    ranges[2 * k + 1] = h->w->ranges()[(size_t)k].end;
  }
}

void fr_warp_interpolated(void* hp, const double* D, int invalid_value, float* out) {
  Handle* h = static_cast<Handle*>(hp);
  cv::Mat wimg;
  h->w->warpImageInterpolated(h->frame, wimg, to_points(D, h->nD), invalid_value);
  std::memcpy(out, wimg.data, sizeof(float) * (size_t)h->nz * h->ny * h->nx);
}

void fr_warp_image(void* hp, const double* D, float* wimg_out, float* cov_out) {
  Handle* h = static_cast<Handle*>(hp);
  cv::Mat wimg, cov;
  h->w->warpImage(h->frame, wimg, cov, to_points(D, h->nD));
  size_t N = (size_t)h->nz * h->ny * h->nx;
  std::memcpy(wimg_out, wimg.data, sizeof(float) * N);
  std::memcpy(cov_out, cov.data, sizeof(float) * N);
}

void fr_warp_point(void* hp, const double* D, int x, int y, int z, int binning, double* out3) {
  Handle* h = static_cast<Handle*>(hp);
  cv::Point3d p = h->w->warpPoint(to_points(D, h->nD), x, y, z, binning);
  out3[0] = p.x;
  out3[1] = p.y;
  out3[2] = p.z;
}

void fr_sobel3d(const float* m, int nz, int ny, int nx, float* gx, float* gy, float* gz) {
  std::vector<int> dims{nz, ny, nx};
  cv::Mat mm = make_mat(m, nz, ny, nx);
  cv::Mat ax(dims, CV_32F), ay(dims, CV_32F), az(dims, CV_32F);
  sobel3d(mm, ax, ay, az);
  size_t N = (size_t)nz * ny * nx;
  std::memcpy(gx, ax.data, N * sizeof(float));
  std::memcpy(gy, ay.data, N * sizeof(float));
  std::memcpy(gz, az.data, N * sizeof(float));
}

// VolumePhaseCorrelator::setReference + computeShift (VolumePhaseCorrelator.cpp:42-139).
void fr_phase_shift(const float* ref, const float* vol, int nz, int ny, int nx, double* shift3) {
  VolumePhaseCorrelator pc(nz, ny, nx);
  pc.setReference(ref);
  cv::Point3d s = pc.computeShift(vol);
  shift3[0] = s.x;
  shift3[1] = s.y;
  shift3[2] = s.z;
}

// The FrameWarpAligner::addFrame solve (FrameWarpAligner.cpp:194-219) with the reference's
// OptimisationModel over the reference warper; rigid shifts are supplied by the caller.
struct ModelCtx {
  OptimisationModel* model;
  int P;
  int evaluations;
};

static double model_f_cb(void* ctx, const double* x) {
  ModelCtx* c = static_cast<ModelCtx*>(ctx);
  column_vector v;
  v.set_size(c->P);
  for (int i = 0; i < c->P; i++) v(i) = x[i];
  c->evaluations++;
  return (*c->model)(v);
}

static void model_g_cb(void* ctx, const double* x, double* g) {
  ModelCtx* c = static_cast<ModelCtx*>(ctx);
  column_vector v, der;
  v.set_size(c->P);
  for (int i = 0; i < c->P; i++) v(i) = x[i];
  dlib::matrix<double> hess;
  c->model->get_derivative_and_hessian(v, der, hess);
  for (int i = 0; i < c->P; i++) g[i] = der(i);
}

static int align_one(Handle* h, const float* frame_data, const double* rigid, int max_iter, double* D_out,
                     int* iters) {
  cv::Mat frame = make_mat(frame_data, h->nz, h->ny, h->nx);
  OptimisationModel model(h->w, frame);
  int nd = h->w->n_dim, P = h->nD * nd;
  ModelCtx ctx{&model, P, 0};
  std::vector<std::vector<double>> start(3, std::vector<double>((size_t)P, 0.0));
  for (int i = 0; i < h->nD; i++)
    for (int c = 0; c < nd; c++) start[2][(size_t)(i * nd + c)] = rigid[c];
  double fe[3];
  for (int s = 0; s < 3; s++) fe[s] = model_f_cb(&ctx, start[(size_t)s].data());
  int best = 0;
  for (int s = 1; s < 3; s++)
    if (fe[s] < fe[best]) best = s;
  std::vector<double> x = start[(size_t)best];
  or_tr_stats st;
  or_trust_region(P, h->w->hess().data(), x.data(), 40.0, 1e-8, max_iter, model_f_cb, model_g_cb, &ctx, &st);
  for (int i = 0; i < h->nD; i++) {
    D_out[3 * i] = x[(size_t)(i * nd)];
    D_out[3 * i + 1] = x[(size_t)(i * nd + 1)];
    D_out[3 * i + 2] = nd == 3 ? x[(size_t)(i * nd + 2)] : 0.0;
  }
  if (iters) *iters = st.iterations;
  return 0;
}

int fr_align_frame(void* hp, const float* frame, const double* rigid, int max_iter, double* D_out, int* iters) {
  return align_one(static_cast<Handle*>(hp), frame, rigid, max_iter, D_out, iters);
}

struct MtJob {
  const float* ref;
  int nz, ny, nx, nD;
  double line, interline, interframe;
  int bidirectional;
  const float* frames;
  const double* rigid;
  int n_frames, max_iter, n_threads, tid;
  double* D_out;
  int* iters;
  Handle* h;
};

static void* mt_worker(void* arg) {
  MtJob* j = static_cast<MtJob*>(arg);
  size_t N = (size_t)j->nz * j->ny * j->nx;
  for (int f = j->tid; f < j->n_frames; f += j->n_threads)
    align_one(j->h, j->frames + (size_t)f * N, j->rigid + 3 * f, j->max_iter, j->D_out + (size_t)f * 3 * j->nD,
              j->iters ? j->iters + f : nullptr);
  return nullptr;
}

// The reference's threading model (FrameAlignerMex.cpp:24-25,120-129: one frame per pool thread).
// CpuFrameWarper keeps an unguarded std::map of error images (FrameWarper.h:158), so each worker
// gets its own warper instance; they are created before the timed call returns control (see
// fr_mt_create) so that fr_mt_align measures alignment only.
void* fr_mt_create(const float* ref, int nz, int ny, int nx, int nD, double line, double interline, double interframe,
                   int bidirectional, int n_threads, char* err) {
  // Warpers are set up in parallel, one per worker thread.
  std::vector<Handle*> hs((size_t)n_threads, nullptr);
  std::vector<pthread_t> th((size_t)n_threads);
  struct Arg {
    const float* ref;
    int nz, ny, nx, nD;
    double line, interline, interframe;
    int bidir;
    Handle** out;
    char err[128];
  };
  std::vector<Arg> args((size_t)n_threads);
  for (int t = 0; t < n_threads; t++) {
    args[(size_t)t] = Arg{ref, nz, ny, nx, nD, line, interline, interframe, bidirectional, &hs[(size_t)t], {0}};
    pthread_create(&th[(size_t)t], nullptr,
                   [](void* p) -> void* {
                     Arg* a = static_cast<Arg*>(p);
                     *a->out = create(a->ref, a->nz, a->ny, a->nx, a->nD, a->line, a->interline, a->interframe,
                                      a->bidir, a->err);
                     return nullptr;
                   },
                   &args[(size_t)t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[(size_t)t], nullptr);
  std::vector<Handle*>* v = new std::vector<Handle*>();
  bool ok = true;
  for (int t = 0; t < n_threads; t++) {
    if (!hs[(size_t)t]) {
      ok = false;
      if (err) std::snprintf(err, 128, "%s", args[(size_t)t].err);
    } else {
      v->push_back(hs[(size_t)t]);
    }
  }
  if (!ok) {
    for (Handle* x : *v) delete x;
    delete v;
    return nullptr;
  }
  return v;
}

void fr_mt_destroy(void* mt) {
  std::vector<Handle*>* v = static_cast<std::vector<Handle*>*>(mt);
  for (Handle* x : *v) delete x;
  delete v;
}

int fr_mt_align(void* mt, const float* frames, int n_frames, const double* rigid, int max_iter, double* D_out,
                int* iters) {
  std::vector<Handle*>* v = static_cast<std::vector<Handle*>*>(mt);
  int n_threads = (int)v->size();
  std::vector<pthread_t> th((size_t)n_threads);
  std::vector<MtJob> jobs((size_t)n_threads);
  for (int t = 0; t < n_threads; t++) {
    Handle* h = (*v)[(size_t)t];
    MtJob j{};
    j.nz = h->nz;
    j.ny = h->ny;
    j.nx = h->nx;
    j.nD = h->nD;
    j.frames = frames;
    j.rigid = rigid;
    j.n_frames = n_frames;
    j.max_iter = max_iter;
    j.n_threads = n_threads;
    j.tid = t;
    j.D_out = D_out;
    j.iters = iters;
    j.h = h;
    jobs[(size_t)t] = j;
    pthread_create(&th[(size_t)t], nullptr, mt_worker, &jobs[(size_t)t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[(size_t)t], nullptr);
  return 0;
}

}  // extern "C"
