/* Stand-in for the generated workspace limit (bytes). */
#define ATL_MaxMalloc 268435456UL
