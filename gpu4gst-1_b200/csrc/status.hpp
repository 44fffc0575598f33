// Thread-local error text behind gst_last_error().
#pragma once
#include <string>

#include "gst_b200.h"

namespace gst {

std::string& last_error_text();

inline gst_status fail(gst_status s, const std::string& msg) {
  last_error_text() = msg;
  return s;
}

}  // namespace gst
