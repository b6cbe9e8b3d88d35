// YUV 4:2:0 planar (I420) frames <-> the codec's FP16 channels-last tensors on the device, so that
// only the 8-bit planes cross PCIe (1.5 bytes per pixel instead of 6).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dcvc {

constexpr int kYuvMaxFrames = 8;

// get_src_frame for YUV 4:2:0 input (test_video.py:69-123 with ycbcr420_to_444_np, transforms.py
// :69-80, nearest-neighbour chroma): src holds `frames` I420 frames back to back (Y H x W, then
// U and V (H/2) x (W/2) each); out[(h * W + w) * ldo + 3 f + c] = FP16(FP16(v / 255) - 0.5) with v
// the Y, U or V sample of frame f (chroma at (h/2, w/2)), the FP16 arithmetic of
// x.half() / 255.0 - 0.5.  H and W even, 1 <= frames <= 8.
cudaError_t launch_yuv420_to_input(const uint8_t* src, int frames, int H, int W, __half* out,
                                   int ldo, cudaStream_t s);

// The reconstruction written by test_video.py (:355-362, yuv_444_to_420 transforms.py:83-90):
// frame f is an FP16 [Hp, Wp, 3] channels-last picture (pixel pitch ldp elements) in
// [-0.5, 0.5], cropped to H x W; x = FP16(x_hat + 0.5); Y = round(clamp(FP16(x * 255), 0, 255));
// U, V = trunc(clamp(FP16(FP16(avg_pool2x2(x)) * 255), 0, 255)) with the pool summed in FP32 in
// row-major order.  dst receives the I420 planes of the frames back to back.
cudaError_t launch_frames_to_yuv420(const __half* const* frames, int nframes, int H, int W, int Wp,
                                    int ldp, uint8_t* dst, cudaStream_t s);

}  // namespace dcvc
