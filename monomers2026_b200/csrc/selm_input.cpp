// selm_input.cpp - reading a reference case directory (placeholder).
#include "selm_engine.h"

int selm_case_create(const char* case_dir, selm_sim** out) {
  (void)case_dir;
  if (out) *out = nullptr;
  return selm_fail(SELM_ERR_IO, "case-directory input is not available in this build");
}
