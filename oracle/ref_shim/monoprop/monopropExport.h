// Stand-in for the CMake-generated export header: symbols keep default visibility.
#pragma once
#define monoprop_EXPORT
#define MONOPROP_EXPORT
