/* Test infrastructure: pre-included (gcc -include) when the reference C is
 * compiled into the "bigtab" oracle build, so that rate tables of up to 1024
 * points fit (the kinetic batch uses 1000-point tables).
 *
 * The reference's include/react_table.h:5-20 fixes MAX_TABLE_SIZE at 500 and
 * defines its guard _REACT_TABLE_H_ after the struct.  This file declares
 * the same struct (same members, same order) with the larger bound and
 * defines the guard first, so the reference's own header becomes empty and
 * every reference source sees this layout.  Nothing else changes. */
#ifndef _REACT_TABLE_H_
#define MAX_TABLE_SIZE 1024

typedef struct react_table react_table;

struct react_table
{
  double e_min;
  double e_step;

  double underflow;
  double overflow;

  int steps;

  double values[MAX_TABLE_SIZE];
};

#define _REACT_TABLE_H_
#endif
