// Stand-in for the QD library's qd_real.h (see dd_real.h beside it).
#pragma once
class qd_real {};
