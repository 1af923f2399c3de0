// tfm_io.hpp -- ITK transform files ("#Insight Transform File V1.0"), the
// format Mirorr reads and writes with itk::TransformFileReader / Writer
// (itkMirorrPyramidWrapper.txx:353-448).
//
//   #Insight Transform File V1.0
//   #Transform 0
//   Transform: Euler3DTransform_double_3_3     (or AffineTransform_double_3_3)
//   Parameters: <6 or 12 values>               (angles x y z + translation, or
//                                               matrix row-major + translation)
//   FixedParameters: <centre x y z>
#pragma once

#include <string>

#include "../../include/mirorr_b200.h"

namespace mirorr_cli {

// Throws std::runtime_error on failure.  The returned transform holds kind,
// params and center (matrix and offset are left for the library to derive).
mirorr_transform read_tfm(const std::string &path);
void write_tfm(const std::string &path, const mirorr_transform &t);

}  // namespace mirorr_cli
