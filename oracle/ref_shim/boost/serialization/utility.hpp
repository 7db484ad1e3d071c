// Empty stand-in (test infrastructure only): frame-aligner's Cv3dUtils.h includes this Boost
// header for cv::Mat serialisation, which the warper path never instantiates.
#pragma once
