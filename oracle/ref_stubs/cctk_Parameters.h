/* Stand-in for the Cactus parameter header.  The only CarpetX parameter the
 * transfer operators read is `prolongate_per_group` (CarpetX/param.ccl:449),
 * which the oracle entry point sets before each call. */
#ifndef CX_REF_STUB_CCTK_PARAMETERS_H
#define CX_REF_STUB_CCTK_PARAMETERS_H
extern int cx_ref_prolongate_per_group;
#define DECLARE_CCTK_PARAMETERS                                                \
  const int prolongate_per_group = cx_ref_prolongate_per_group;                \
  (void)prolongate_per_group;
#endif
