// Host-side pieces of the DDM engine that need no GPU: annulus masks, the reference's
// chunk schedule, parameter validation and the ISF text format.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ddm {

constexpr int kLabelUninit = -1;  // ring data the reference never wrote

// q radius in spectrum pixels for scale s and wavelength lambda, in IEEE single
// precision: static_cast<float>(scale) / lambda (src/DDM.cu:102).
float q_radius(int scale, float lambda);

// Annulus masks of one scale, bit-exact to buildAzimuthMask
// (src/azimuthal_average.cu:229-283): for kx in [0, s/2], ky in [0, s), signed
// frequencies x' = (kx + s/2) % s - s/2 (same for y), r2 = float(x'^2 + y'^2),
// pixel in mask q iff 1 <= r2 / (q*q) <= tol*tol, every step in float.
// Emits, per q, the sorted element indices ky*(s/2+1) + kx (CSR) and the counts.
void build_masks(int scale, const std::vector<float> &lambdas, float tolerance,
                 std::vector<int> *q_ptr, std::vector<int> *idx, std::vector<int> *counts);

// One iteration of the reference's chunk loop (src/DDM.cu:765-843) on frame labels:
// the A frames are start[fo] for fo < count, and the partner of (fo, tau) is
// position p = fo + tau of the concatenation start|end.
struct CompatIteration {
    std::vector<int> start;  // C labels
    std::vector<int> end;    // C labels
    int count = 0;           // frame offsets analysed (C, or L for the leftover pass)
    bool dump_after = false; // -G snapshot + purge after this iteration (src/DDM.cu:800)
    int min_label = 0, max_label = -1;  // over the labels this iteration reads
};

// Replays src/DDM.cu:750-843 with labels instead of pixels. `frames_read` is how many
// frames the reference reads from its source (at least 2C).
std::vector<CompatIteration> compat_schedule(int total_frames, int chunk, int multistream,
                                             int dump_every, const std::vector<int> &taus,
                                             int *frames_read);

// Parameter checks of runDDM (src/DDM.cu:327-355, 459-463) on sorted arrays. Returns an
// empty string when valid, else the reference's message. `warnings` collects the
// reference's non-fatal messages.
std::string validate_reference_params(const std::vector<int> &scales, const std::vector<int> &taus,
                                      const std::vector<float> &lambdas, float tolerance,
                                      int chunk, bool enforce_tau_chunk,
                                      bool enforce_lambda_scale, std::vector<std::string> *warnings);

// writeIqtToFile (src/azimuthal_average.cu:112-150) text layout.
bool write_isf_file(const std::string &path, const double *isf_qt, const std::vector<float> &lambdas,
                    const std::vector<int> &taus, float fps);

}  // namespace ddm
