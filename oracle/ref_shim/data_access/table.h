/* Stand-in for the reference's data_access/table.h: intermediate.h includes
 * it, but nothing on the execute() path uses the Table loader, which needs
 * range-v3. TEST INFRASTRUCTURE. */
#pragma once
#include <data_model/plan.h>
