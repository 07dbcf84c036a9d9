// Internal declarations shared by the host compile and the device runtime.
#pragma once
#include <array>
#include <map>
#include <string>
#include <vector>

#include "../../include/grico_b200.h"

namespace grico {
void set_error(const std::string& msg);
void fe_basis(double x, int p, double* v, double* d);
void gauss_legendre(int count, double* pts, double* wts);
std::vector<double> affine_restriction_matrix(int src_deg, int tgt_deg, int delta, long long rel);
}  // namespace grico
