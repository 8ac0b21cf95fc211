// Header-only stand-in for the boost pieces the reference path includes.
// Test infrastructure only: lets the reference's own sources compile with g++
// where boost is not installed. No arithmetic of the traced path lives here.
#pragma once
#include <memory>
#include <cassert>
#ifndef BOOST_ASSERT
#define BOOST_ASSERT(x) assert(x);
#endif
namespace boost { using std::shared_ptr; using std::make_shared; using std::dynamic_pointer_cast; using std::static_pointer_cast; }
