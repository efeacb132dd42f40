// status.hpp — the mapping of C++ exceptions to the C8R_* status codes of
// include/c8radio.h, shared by every file that defines extern "C" entry
// points.  Each reference exception class has its own code, so the C++ shim
// (include/c8radio.hpp) can throw the same class again.
#pragma once

#include <new>
#include <stdexcept>
#include <string>

#include "../../include/c8radio.h"

namespace c8r {

// A failing CUDA runtime call (C8R_CUDA_ERROR rather than C8R_RUNTIME_ERROR,
// which stands for the reference's fixed-point overflow at download).
struct cuda_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Runs `body`; returns C8R_OK, or the status of the exception it threw with
// its message stored in *error (when error is not null).
template <class F>
int guarded(std::string* error, F&& body) {
  try {
    body();
    return C8R_OK;
  } catch (std::invalid_argument const& e) {
    if (error) *error = e.what();
    return C8R_INVALID_ARGUMENT;
  } catch (std::out_of_range const& e) {
    if (error) *error = e.what();
    return C8R_OUT_OF_RANGE;
  } catch (std::length_error const& e) {
    if (error) *error = e.what();
    return C8R_LENGTH_ERROR;
  } catch (std::logic_error const& e) {
    if (error) *error = e.what();
    return C8R_LOGIC_ERROR;
  } catch (std::overflow_error const& e) {
    if (error) *error = e.what();
    return C8R_OVERFLOW_ERROR;
  } catch (cuda_error const& e) {
    if (error) *error = e.what();
    return C8R_CUDA_ERROR;
  } catch (std::runtime_error const& e) {
    if (error) *error = e.what();
    return C8R_RUNTIME_ERROR;
  } catch (std::bad_alloc const&) {
    if (error) *error = "radio allocation failed";
    return C8R_BAD_ALLOC;
  } catch (...) {
    if (error) *error = "unknown radio failure";
    return C8R_RUNTIME_ERROR;
  }
}

// Message slot of entry points without a handle (c8r_last_global_error).
void set_global_error(char const* message);

}  // namespace c8r
