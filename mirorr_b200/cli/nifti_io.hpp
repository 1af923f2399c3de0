// nifti_io.hpp -- NIfTI-1 volumes (.nii, .nii.gz) in ITK's conventions.
//
// Reading converts any scalar datatype to float32 (scl_slope / scl_inter
// applied) and the header's orientation to ITK's LPS physical frame, as
// itk::NiftiImageIO does: the voxel-to-RAS transform comes from the qform
// (qform_code > 0), else the sform (sform_code > 0), else the pixel spacing;
// spacing is the column norms, direction the normalised columns, and the
// first two rows of direction and origin change sign (RAS -> LPS).
// Writing stores float32 or uint8 with matching qform and sform (code 1).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mirorr_b200.h"

namespace mirorr_cli {

struct Volume {
  mirorr_geometry geom{};   // ITK geometry (LPS)
  std::vector<float> data;  // x fastest
};

// Throws std::runtime_error with the file name on failure.
Volume read_nifti(const std::string &path);
void write_nifti_float(const std::string &path, const mirorr_geometry &g, const float *data);
void write_nifti_u8(const std::string &path, const mirorr_geometry &g, const uint8_t *data);

}  // namespace mirorr_cli
