#pragma once
#include "ptime.hpp"
