// What the host request layer (nf_server.cu) needs to know about a plan: its temporal
// configuration and which launch forms accept it. Implemented beside the plan (nf_api.cu).
#pragma once
#include "neo_fft_b200.h"

namespace nfi {

struct PlanInfo {
  bool fft3d = false;
  int width = 0, height = 0, elem = 1;  // plane size, bytes per sample
  int temporal_size = 1;
  bool tmode1 = false;                  // DFTTest temporal overlap-add (tmode 1)
  int temporal_overlap = 0;
  bool kalman = false, preview = false;
  bool single = false;  // accepted by nf_batch (single-frame filter)
  bool clip = false;    // accepted by nf_clip_batch
  int pframe = 0;       // FFT3D pattern frame (pfactor)
  int kalman_warmup = 8;  // FFT3D bt=0: frames replayed at most before a random-access request
  int device = 0;         // CUDA device the plan's tables live on
};

PlanInfo plan_info(const nf_plan* p);

// The checks nf_dft_backward_device applies to its plan and plane count (a float DFTTest
// plan with tbsize 1, smode 1 and ftype 0..2; 1..32 planes), as a status and message.
nf_status check_backward_call(const nf_plan* p, int nplanes, char* err, size_t len);

}  // namespace nfi
