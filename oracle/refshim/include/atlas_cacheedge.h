/* Stand-in for the generated L2 blocking edge (bytes). */
#define CacheEdge 262144
