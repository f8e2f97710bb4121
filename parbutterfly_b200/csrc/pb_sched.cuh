// Learned scheduler, peeling side (pb_sched.cu).
#pragma once

#include "pb_engine.cuh"
#include "pb_mlp.cuh"

namespace pb {

constexpr int kPeelCallFeatures = 12;  // call-level features; 4 candidate slots follow
constexpr int kWingCandidates = 3;     // 3 work-unit counts (full grid, one round at a time)
constexpr int kTipCandidates = 48;     // 3 round batchings x 4 grid-level thresholds x 4 CTA counts

int peel_candidates(bool wing);
// Work-unit setting c of the candidate grid of a peel kind (c = 0: the plain path's setting);
// resident_ctas is the CTA count of a full persistent launch.
PeelTuning peel_candidate(bool wing, int c, int resident_ctas);
// Call-level features of a peel call (kPeelCallFeatures floats into f).
void peel_call_features(const pb_graph& g, int use_v, bool wing, const int64_t* counts_dev, float* f, cudaStream_t s);
// Cost-model row of candidate c for a call (kMlpIn floats).
void peel_row(const float* call_f, bool wing, int c, float* row);
// The candidate with the least predicted log2(ms); its prediction in *pred_log2ms.
int choose_peel(MlpModel& model, const float* call_f, bool wing, float* pred_log2ms, cudaStream_t s);

}  // namespace pb
