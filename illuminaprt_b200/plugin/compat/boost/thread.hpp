#pragma once
#include "thread/thread.hpp"
#include "thread/tss.hpp"
#include "thread/recursive_mutex.hpp"
