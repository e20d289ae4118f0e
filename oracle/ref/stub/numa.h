/* TEST INFRASTRUCTURE ONLY: libnuma's <numa.h> is absent here; the reference's
 * sorting/affinity sources include it but call nothing from it in the paths
 * that the harness runs (one NUMA node). */
#pragma once
