// TEST INFRASTRUCTURE ONLY: see Partio.h in this directory.
#pragma once
#include "Partio.h"
