// Stand-in for the QD library's dd_real.h, which is not installed: the
// reference's qdldl-luir/tblas.hpp includes it unconditionally but the
// harness instantiates its templates with float and double only.
#pragma once
class dd_real {};
