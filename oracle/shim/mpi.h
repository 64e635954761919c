#include "petsc.h"
