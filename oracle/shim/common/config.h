/* Empty build-configuration header for the reference runtime (oracle build only). */
