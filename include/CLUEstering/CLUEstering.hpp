// Drop-in umbrella header: code written against CLUEstering's
// `#include "CLUEstering/CLUEstering.hpp"` gets the libclue_sm100 API
// (namespace clue) with the same class and function names.
#pragma once
#include "../clue_sm100.hpp"
