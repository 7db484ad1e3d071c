// B200FrameWarper.h -- the drop-in warper for flimfit/frame-aligner: an AbstractFrameWarper
// (FrameAligner/FrameWarper.h:95-143) over this library's C ABI (include/fa_b200.h), in place of
// GpuFrameWarper (FrameAligner/GpuFrameWarper.h:31-72).
//
// A maintainer copies this header into FrameAligner/, adds include/ to the include path, links
// frame-aligner_b200/libfa_b200.so and selects the class where FrameWarpAligner picks its warper
// (FrameAligner/FrameWarpAligner.cpp:14-27). It compiles against the reference's own headers and
// OpenCV / dlib types: frames are CV_32F, continuous, {nz, ny, nx}, identified by their data pointer
// like GpuFrameWarper's (GpuFrameWarper.h:55); library errors become std::runtime_error, as the
// reference reports its own.
#pragma once

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "FrameWarper.h"
#include "GpuFrameWarper.h"  // GpuSupportInformation (GpuFrameWarper.h:5-17)
#include "fa_b200.h"

class B200FrameWarper : public AbstractFrameWarper
{
public:
   explicit B200FrameWarper(int device = 0, fa_precision precision = FA_PREC_F32) : precision(precision)
   {
      fa_config cfg = {device, 0, 0};
      check(fa_create(&cfg, &ctx));
   }

   ~B200FrameWarper()
   {
      for (auto& f : frames) fa_deregister_frame(f.second);
      if (ref) fa_reference_destroy(ref);
      fa_destroy(ctx);
   }

   B200FrameWarper(const B200FrameWarper&) = delete;
   B200FrameWarper& operator=(const B200FrameWarper&) = delete;

   // GpuFrameWarper::getGpuSupportInformation (GpuFrameWarper.cpp:16-44)
   static GpuSupportInformation getGpuSupportInformation()
   {
      int ok = 0;
      char msg[256] = {0};
      if (fa_gpu_support(&ok, msg, sizeof(msg)) != FA_OK) return GpuSupportInformation(false, fa_last_error());
      return GpuSupportInformation(ok != 0, msg);
   }

   // Sum of squared errors (CpuFrameWarper::getError, FrameWarper.cpp:169-176)
   double getError(const cv::Mat& img, const std::vector<cv::Point3d>& D) override
   {
      double f = 0;
      check(fa_get_error(frame(img), points(D), &f));
      return f;
   }

   // J^T e (AbstractFrameWarper::computeJacobian, FrameWarper.cpp:147-167), P = nD * n_dim
   void getJacobian(const cv::Mat& img, const std::vector<cv::Point3d>& D, column_vector& jac) override
   {
      jac.set_size(nD * n_dim);
      check(fa_get_jacobian(frame(img), points(D), &jac(0)));
   }

   // CpuFrameWarper::warpImageInterpolated (FrameWarper.cpp:31-69)
   void warpImageInterpolated(const cv::Mat& img, cv::Mat& wimg, const std::vector<cv::Point3d>& D,
                              int invalid_value = 0) override
   {
      wimg = cv::Mat(dims, CV_32F);
      check(fa_warp(frame(img), points(D), (float) invalid_value, (float*) wimg.data));
   }

   // GpuFrameWarper::registerFrame / deregisterFrame (GpuFrameWarper.cpp:46-73)
   void registerFrame(const cv::Mat& f) override
   {
      if (!ref) throw std::runtime_error("Reference imaging not yet set");
      fa_frame* h = nullptr;
      check(fa_register_frame(ref, f.data, FA_F32, &h));
      std::lock_guard<std::mutex> lk(mutex);
      auto it = frames.find(f.data);
      if (it != frames.end()) fa_deregister_frame(it->second);
      frames[f.data] = h;
   }

   void deregisterFrame(const cv::Mat& f) override
   {
      std::lock_guard<std::mutex> lk(mutex);
      auto it = frames.find(f.data);
      if (it != frames.end())
      {
         fa_deregister_frame(it->second);
         frames.erase(it);
      }
   }

protected:
   // Called at the end of AbstractFrameWarper::setReference (FrameWarper.cpp:186-205), after the
   // reference's own CPU tables are built: the device set-up builds what the library needs and
   // fills H, which OptimisationModel reads (OptimisationModel.cpp:55-62).
   void setupReferenceInformation() override
   {
      {
         std::lock_guard<std::mutex> lk(mutex);
         for (auto& f : frames) fa_deregister_frame(f.second);
         frames.clear();
      }
      if (ref) fa_reference_destroy(ref);
      ref = nullptr;
      fa_scan_params sp = {image_params.line_duration, image_params.interline_duration,
                           image_params.pixel_duration, image_params.frame_duration,
                           image_params.interframe_duration, image_params.stack_duration,
                           image_params.n_x, image_params.n_y, image_params.n_z,
                           image_params.bidirectional ? 1 : 0};
      cv::Mat r = reference.isContinuous() ? reference : reference.clone();
      check(fa_set_reference(ctx, (const float*) r.data, dims[0], dims[1], dims[2], nD, &sp, precision, &ref));
      H.set_size(nD * n_dim, nD * n_dim);
      check(fa_get_hessian(ref, &H(0, 0)));
   }

private:
   static void check(fa_status s)
   {
      if (s != FA_OK) throw std::runtime_error(fa_last_error());
   }

   // std::vector<cv::Point3d> is nD x 3 contiguous doubles, the layout the C ABI takes
   const double* points(const std::vector<cv::Point3d>& D) const
   {
      if ((int) D.size() != nD) throw std::runtime_error("D has the wrong number of control points");
      return &D[0].x;
   }

   fa_frame* frame(const cv::Mat& img)
   {
      std::lock_guard<std::mutex> lk(mutex);
      auto it = frames.find(img.data);
      if (it == frames.end()) throw std::runtime_error("Unrecognised frame");  // GpuFrameWarper.cpp:162-167
      return it->second;
   }

   fa_precision precision;
   fa_context* ctx = nullptr;
   fa_reference* ref = nullptr;
   std::map<void*, fa_frame*> frames;
   std::mutex mutex;
};
