// scheme.h -- filter weights shared by the host tables and the device kernels.
//
// The Vasilyev-Lund-Moin 7-point xi/eta filter and the Hanasoge-Duvall 11-point radial
// filter, centre weight first, as the reference lists them (header:99-105, 123-133).
// They are compile-time values so that the filter kernel takes them as immediates.
#pragma once

namespace solar {

constexpr double kFilt[4] = {0.6875, 0.234375, -0.09375, 0.015625};
constexpr double kFiltR[6] = {0.753906, 0.2050775, -0.1171875, 0.043945, -0.0097655, 0.0009765};

}  // namespace solar
