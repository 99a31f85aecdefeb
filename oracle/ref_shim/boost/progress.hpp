// Build-only stand-in for boost::progress_display, the one Boost facility
// the reference CLI uses (a console progress bar). It draws nothing; the
// reference's results do not depend on it.
#pragma once
#include <cstddef>
namespace boost {
struct progress_display {
    explicit progress_display(std::size_t) {}
    progress_display &operator++() { return *this; }
};
}
