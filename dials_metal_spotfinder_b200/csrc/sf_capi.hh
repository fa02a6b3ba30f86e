// Exception-to-status translation shared by the C entry points.
#pragma once

#include <stdexcept>

#include "sf_host.hh"

namespace sf {

// A labelling input the reference would refuse with std::runtime_error
// (frame out of order, pixels not ascending, pixel off the frame): -4.
struct Refused : std::runtime_error {
  using std::runtime_error::runtime_error;
};

template <typename F> int guarded(F &&body) {
  try {
    return body();
  } catch (const DeviceError &e) {
    set_error(e.what());
    return -3;
  } catch (const Refused &e) {
    set_error(e.what());
    return -4;
  } catch (const std::invalid_argument &e) {
    set_error(e.what());
    return -1;
  } catch (const std::out_of_range &e) {
    set_error(e.what());
    return -1;
  } catch (const std::exception &e) {
    set_error(e.what());
    return -3;
  }
}

} // namespace sf
