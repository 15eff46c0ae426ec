// InvMR lives with the other single-shift solvers.
#pragma once
#include "qphix/invcg.h"
