# qualify.sed -- the one source change the reference's applications need to
# run on the GPU engine: IP_DEVICE on the functions that become device code,
# IP_GLOBAL on the file-scope variables that ip_compute reads.
s/^void ip_compute(/IP_DEVICE void ip_compute(/
s/^void ip_combine(/IP_DEVICE void ip_combine(/
s/^double ratio;/IP_GLOBAL double ratio;/
s/^double initial_value;/IP_GLOBAL double initial_value;/
s/^IP_VERTEX_ID_TYPE start_vertex;/IP_GLOBAL IP_VERTEX_ID_TYPE start_vertex;/
