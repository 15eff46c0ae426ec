// tm_clov_dslash_def.h: the drop-in Dslash family lives in qphix/dslash_def.h.
#pragma once
#include "qphix/dslash_def.h"
